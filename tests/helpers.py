"""Shared test inputs: seeded molecules, their QUICK arrays and densities."""
import numpy as np

from quick_b200.basis import build_basis
from quick_b200.molecule import linear_alkane, water_cluster

CASES = {
    "water2_631gs": (lambda: water_cluster((2, 1, 1), seed=0), "6-31G*"),
    "water4_631gs": (lambda: water_cluster((2, 2, 1), seed=0), "6-31G*"),
    "water3_631gss": (lambda: water_cluster((3, 1, 1), seed=2), "6-31G**"),
    "propane_631gss": (lambda: linear_alkane(3, seed=1), "6-31G**"),
    "hexane_631gs": (lambda: linear_alkane(6, seed=4), "6-31G*"),
}


def case(name):
    mk, bas = CASES[name]
    m = mk()
    return m, build_basis(m.symbols, bas)


def random_density(n, seed=0, scale=0.1):
    """A symmetric test density with entries spread like a real one."""
    rng = np.random.default_rng(seed)
    d = rng.standard_normal((n, n)) * scale
    d = d + d.T
    d[np.diag_indices(n)] += 1.0
    return np.asfortranarray(d)


def psd_density(n, nocc, seed=0, scale=0.3):
    """A positive semi-definite closed-shell density 2 C C^T (so rho(r) >= 0
    everywhere, as for a real density), C random (n x nocc)."""
    rng = np.random.default_rng(seed)
    c = rng.standard_normal((n, nocc)) * scale
    return np.asfortranarray(2.0 * c @ c.T)


# QUICK's published HF total energies for its ACE-(ALA)n-NME benchmark inputs
# (info/quick.cuda_benchmark.numbers, "Table 1-1", GPU column, Eh; the sheet's
# rows matched to the input files by their basis-function counts).  Only the
# rows for ala2.in and ala3.in are the molecules of the files: the rows
# matched to ala1.in and ala5.in have the right basis-function counts but
# energies several mEh (ala1) and 0.13 Eh (ala5, 6-31G*) away from any SCF
# solution of those geometries, so the sheet computed other structures there.
PUBLISHED_HF = {
    ("ala2", "6-31G"): -492.557816881,
    ("ala2", "6-31G*"): -492.781504479,
    ("ala3", "6-31G"): -738.266673086,
    ("ala3", "6-31G*"): -738.604777138,
}


def ace_ala(name):
    """An ACE-(ALA)n-NME molecule from QUICK's benchmark inputs
    (tests/golden/ace_ala_nme.json, written by make_ace_ala.py)."""
    import json
    import os
    from quick_b200.molecule import Molecule
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "ace_ala_nme.json")) as fh:
        d = json.load(fh)[name]
    return Molecule(d["symbols"], np.array(d["xyz_angstrom"]))


class OracleEngine:
    """The SCF engine interface of quick_b200.scf over the CPU oracle:
    one-electron integrals, QUICK's Fock build and the full gradient."""

    def __init__(self, mol, basis, integral_cutoff=1e-10, prim_limit=1e-20, method=0):
        import oracle
        self.o = oracle
        self.mol, self.basis = mol, basis
        self.cut, self.plim = integral_cutoff, prim_limit
        self.Y, self.cp = oracle.schwarz(basis, mol.xyz_bohr)
        # 0 HF, 1 B3LYP (exchange fraction 0.2), 2 BLYP; the functional from
        # QUICK's own getxc compiled for the host
        self.method = method
        self.hybrid = {0: 1.0, 1: 0.2, 2: 0.0}[method]
        if method:
            from quick_b200.basis import sigrad2
            self.sg = sigrad2(basis)
            self._keep = oracle.ref_upload_molecule(mol, basis, self.Y, self.cp)

    def xc(self, D):
        n = self.basis.nbasis
        V, exc, _, _ = self.o.ref_getxc(np.zeros((n, n), order="F"), D, self.sg, method=self.method)
        return V, exc

    def overlap_core(self):
        return self.o.oneint(self.basis, self.mol)

    def enuc(self):
        return self.o.enuc(self.mol)

    def fock2e(self, D):
        G, _ = self.o.fock(self.basis, self.mol.xyz_bohr, self.Y, self.cp, self.o.cutmatrix(self.basis, D), D,
                           self.cut, self.plim, hybrid=self.hybrid)
        return G

    def gradient(self, D, W):
        g = self.o.grad1e(self.basis, self.mol, D, W)
        return g + self.o.grad2e(self.basis, self.mol.xyz_bohr, self.Y, self.cp, self.o.cutmatrix(self.basis, D), D,
                                 self.cut, self.plim)
