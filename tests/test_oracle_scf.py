"""The one-electron oracle and the SCF driver on the CPU: literature HF
energies, QUICK's published energy for ACE-(ALA)2-NME, the same SCF with
QUICK's own two-electron kernels (host build), and the full analytic gradient
against central finite differences of the SCF energy."""
import math

import numpy as np
import pytest

from helpers import PUBLISHED_HF, OracleEngine, ace_ala
from quick_b200 import scf
from quick_b200.basis import A_TO_BOHRS, build_basis
from quick_b200.molecule import Molecule


def _water(r=0.947, theta=105.5):
    t = math.radians(theta)
    return Molecule(["O", "H", "H"], np.array([[0, 0, 0], [r, 0, 0], [r * math.cos(t), r * math.sin(t), 0]]))


def _rhf(m, bs, cut=1e-12, conv=1e-9):
    b = build_basis(m.symbols, bs)
    eng = OracleEngine(m, b, cut, 1e-25)
    return scf.rhf(eng, m.n_electrons // 2, conv=conv), eng, b


def test_literature_energies(oracle_lib):
    """Textbook HF energies: H2 at R = 1.4 bohr in 6-31G (-1.1268) and
    6-31G** (-1.1313) (Szabo & Ostlund, Modern Quantum Chemistry, chapter 3),
    and H2O at its HF/6-31G* optimum r = 0.947 A, 105.5 deg (-76.010746)."""
    R = 1.4 / A_TO_BOHRS
    h2 = Molecule(["H", "H"], np.array([[0, 0, 0], [0, 0, R]]))
    r1, _, _ = _rhf(h2, "6-31G")
    r2, _, _ = _rhf(h2, "6-31G**")
    rw, _, _ = _rhf(_water(), "6-31G*")
    assert r1.converged and r2.converged and rw.converged
    assert abs(r1.energy - -1.1268) < 1e-4
    assert abs(r2.energy - -1.1313) < 1e-4
    assert abs(rw.energy - -76.010746) < 2e-6


def test_overlap_and_core_properties(oracle_lib):
    """S is symmetric with unit diagonal on the s and p functions (QUICK
    normalises x^2-type components), positive definite; the one-electron
    matrices are symmetric; nuclear repulsion matches the Molecule's."""
    m = _water()
    b = build_basis(m.symbols, "6-31G*")
    S, H = oracle_lib.oneint(b, m)
    assert np.abs(S - S.T).max() == 0.0 and np.abs(H - H.T).max() == 0.0
    sp = np.array([sum(b.itype[:, i]) <= 1 for i in range(b.nbasis)])
    assert np.allclose(np.diag(S)[sp], 1.0, atol=1e-12)
    assert np.linalg.eigvalsh(S).min() > 1e-3
    assert abs(oracle_lib.enuc(m) - m.nuclear_repulsion()) < 1e-12


def test_cut_matrix_matches_oracle(oracle_lib):
    m = _water()
    b = build_basis(m.symbols, "6-31G*")
    rng = np.random.default_rng(1)
    D = rng.standard_normal((b.nbasis, b.nbasis))
    D = D + D.T
    assert np.array_equal(scf.shell_cut_matrix(b, D), oracle_lib.cutmatrix(b, D))


def test_orthogonaliser():
    rng = np.random.default_rng(2)
    a = rng.standard_normal((12, 12))
    S = a @ a.T + 12 * np.eye(12)
    X = scf.orthogonaliser(S)
    assert np.allclose(X.T @ S @ X, np.eye(12), atol=1e-12)


def test_full_gradient_vs_finite_differences(oracle_lib):
    """Analytic RHF gradient (one-electron + nuclear + two-electron) against
    central differences of the converged SCF energy, h = 1e-3 bohr."""
    m = _water(0.96, 103.0)
    r, eng, b = _rhf(m, "6-31G*", conv=1e-10)
    g = eng.gradient(r.D, r.W)
    h = 1e-3
    for atom, k in ((0, 0), (1, 1), (2, 0), (2, 1)):
        xs = []
        for sgn in (1, -1):
            x = m.xyz_angstrom.copy()
            x[atom, k] += sgn * h / A_TO_BOHRS
            xs.append(_rhf(Molecule(m.symbols, x), "6-31G*", conv=1e-10)[0].energy)
        fd = (xs[0] - xs[1]) / (2 * h)
        assert abs(g[3 * atom + k] - fd) < 1e-6, (atom, k, g[3 * atom + k], fd)
    # translational invariance of the analytic gradient
    assert np.abs(g.reshape(-1, 3).sum(axis=0)).max() < 1e-9


def test_ala2_published_energy(oracle_lib):
    """ACE-(ALA)2-NME in 6-31G with QUICK's keywords (cutoff 1e-9, density
    RMS 1e-8).  QUICK's published energy (2011) is 1.0e-5 Eh above this
    code's; QUICK's present two-electron kernels give this code's value (next
    test), so the difference lies outside the two-electron path."""
    m = ace_ala("ala2")
    b = build_basis(m.symbols, "6-31G")
    r = scf.rhf(OracleEngine(m, b, 1e-9, 1e-20), m.n_electrons // 2, conv=1e-8)
    assert r.converged
    assert abs(r.energy - PUBLISHED_HF[("ala2", "6-31G")]) < 2e-5
    assert abs(r.energy - -492.557827108) < 2e-9


def test_scf_with_quicks_own_kernels():
    """The same SCF with QUICK's own get2e kernels (compiled for the host)
    in place of the oracle's Fock build gives the same energy."""
    import oracle
    if not oracle.ref_available():
        pytest.skip("QUICK's host build (oracle/_ref) not available")
    m = ace_ala("ala2")
    b = build_basis(m.symbols, "6-31G")
    eng = OracleEngine(m, b, 1e-9, 1e-20)
    oracle.ref_upload_molecule(m, b, eng.Y, eng.cp, threads=16)

    class QuickEngine(OracleEngine):
        def fock2e(self, D):
            n = b.nbasis
            return oracle.ref_get2e(np.zeros((n, n), order="F"), D, oracle.cutmatrix(b, D), 1e-9, 1e-20)

    qe = QuickEngine(m, b, 1e-9, 1e-20)
    r = scf.rhf(qe, m.n_electrons // 2, conv=1e-8)
    assert r.converged
    assert abs(r.energy - -492.557827108) < 1e-8


def test_sad_guess(oracle_lib):
    """The superposition-of-atomic-densities guess holds the molecule's
    electrons (tr DS = N) and the SCF from it reaches the core guess's energy."""
    from quick_b200.molecule import water_cluster
    m = water_cluster((2, 1, 1), seed=4)
    b = build_basis(m.symbols, "6-31G*")

    def atom_density(sym):
        a = Molecule([sym], np.zeros((1, 3)))
        ab = build_basis(a.symbols, "6-31G*")
        r = scf.rhf(OracleEngine(a, ab, 1e-12, 1e-20), a.n_electrons / 2.0, conv=1e-7, max_iter=60, fractional=True)
        assert r.converged
        return r.D

    D0 = scf.sad_guess(m, b, atom_density)
    S, _ = oracle_lib.oneint(b, m)
    assert abs(np.sum(D0 * S) - m.n_electrons) < 1e-8
    eng = OracleEngine(m, b, 1e-11, 1e-20)
    r_sad = scf.rhf(eng, m.n_electrons // 2, conv=1e-9, D0=D0)
    r_core = scf.rhf(eng, m.n_electrons // 2, conv=1e-9)
    assert r_sad.converged and r_core.converged
    assert abs(r_sad.energy - r_core.energy) < 1e-9
    assert r_sad.iterations <= r_core.iterations


def test_aufbau_occupations():
    occ = scf.aufbau_occupations(np.array([-1.0, -0.5, -0.2, -0.2, -0.2, 0.3]), 7)
    assert np.allclose(occ, [2, 2, 1, 1, 1, 0])
    occ = scf.aufbau_occupations(np.array([-1.0, -0.5]), 3)
    assert np.allclose(occ, [2, 1])


def test_kohn_sham_oracle_scf():
    """The oracle's Kohn-Sham SCF (QUICK's own getxc on the host) converges,
    reproduces the committed value and lies within a few mEh of the
    literature B3LYP/6-31G* water energy (about -76.409 near this geometry)."""
    import json
    import os
    import oracle
    if not oracle.ref_available():
        pytest.skip("QUICK's host build (oracle/_ref) not available")
    with open(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "scf_golden.json")) as fh:
        gold = json.load(fh)["energies"]
    t = math.radians(104.5)
    m = Molecule(["O", "H", "H"], np.array([[0, 0, 0], [0.96, 0, 0], [0.96 * math.cos(t), 0.96 * math.sin(t), 0]]))
    b = build_basis(m.symbols, "6-31G*")
    r = scf.rhf(OracleEngine(m, b, 1e-11, 1e-20, method=1), m.n_electrons // 2, conv=1e-8)
    assert r.converged
    assert abs(r.energy - gold["water/6-31G*/B3LYP"]) < 1e-9
    assert abs(r.energy - -76.409) < 5e-3
