"""Closed-shell SCF driver around the GPU Fock build and gradient.

QUICK's own Fortran host (``getEnergy`` in src/getEnergy.f90, the DIIS SCF
``electdiis`` in src/scf.f90:60-650, ``fullx`` in
src/quick_one_electron_integral.f90:18-126 and ``hfgrad`` in
src/gradient.f90) calls the ``gpu_*`` entry points once per iteration.  This
module plays that host's part so that total energies and full nuclear
gradients can be formed and timed: it orthogonalises with S^-1/2, iterates
Roothaan-Hall with Pulay DIIS until the density RMS change falls below the
requested threshold, and forms the energy-weighted density for the gradient.

The integrals come from an *engine* object:

* ``overlap_core()`` -> (S, H), the overlap and core Hamiltonian;
* ``fock2e(D)``      -> G(D), the two-electron part of the Fock matrix;
* ``enuc()``         -> the nuclear repulsion energy;
* ``gradient(D, W)`` -> the full nuclear gradient (3 natom).

``GpuEngine`` binds them to this package's C ABI (one-electron integrals,
Fock build and gradients on the GPU).  With ``incremental=True`` the Fock
matrix is updated with G(D_n - D_n-1), whose density screen discards more
quartets as the SCF converges, and rebuilt in full every ``rebuild_every``
iterations.
"""
import time
from dataclasses import dataclass, field

import numpy as np


def shell_cut_matrix(basis, D):
    """QUICK's density screen cutMatrix(II,JJ) = max |D| over the shell-pair
    block (src/schwarz.f90:550-599)."""
    first = basis.Ksumtype[:-1] - 1
    last = basis.Ksumtype[1:] - 1
    A = np.abs(D)
    rowmax = np.stack([A[f:l].max(axis=0) for f, l in zip(first, last)])   # (nshell, nbasis)
    cm = np.stack([rowmax[:, f:l].max(axis=1) for f, l in zip(first, last)], axis=1)
    return np.asfortranarray(np.maximum(cm, cm.T))


def orthogonaliser(S, threshold=1e-4):
    """X with X^T S X = 1: S^-1/2 over the eigenvectors of S whose eigenvalue
    exceeds ``threshold`` (fullx drops the others, :78-85)."""
    s, U = np.linalg.eigh(S)
    keep = s > threshold
    if keep.all():
        return (U * s ** -0.5) @ U.T
    return U[:, keep] * s[keep] ** -0.5


@dataclass
class SCFResult:
    energy: float                 # total energy, Eh
    e_elec: float
    e_nuc: float
    converged: bool
    iterations: int
    D: np.ndarray                 # total density of the last Fock build
    C: np.ndarray                 # MO coefficients
    eps: np.ndarray               # orbital energies
    nocc: int
    history: list = field(default_factory=list)   # per iteration: (energy, drms, seconds)
    fock_seconds: float = 0.0
    seconds: float = 0.0

    @property
    def W(self):
        """Energy-weighted density 2 sum_occ e_k C_k C_k^T (gradient.f90:84-96)."""
        Co = self.C[:, :self.nocc]
        return 2.0 * (Co * self.eps[:self.nocc]) @ Co.T


def _density(C, nocc):
    Co = C[:, :nocc]
    return 2.0 * Co @ Co.T


def aufbau_occupations(eps, nelec, tol=1e-4):
    """Occupation numbers for ``nelec`` electrons over orbital energies
    ``eps`` (ascending): two per orbital, the last partly filled degenerate
    set (energies within ``tol``) shared equally, which keeps an atom's
    density spherical."""
    occ = np.zeros(len(eps))
    left = float(nelec)
    i = 0
    while left > 1e-12 and i < len(eps):
        j = i
        while j + 1 < len(eps) and eps[j + 1] - eps[i] < tol:
            j += 1
        g = j - i + 1
        put = min(left, 2.0 * g)
        occ[i:j + 1] = put / g
        left -= put
        i = j + 1
    return occ


def rhf(engine, nocc, conv=1e-8, max_iter=100, diis_size=10, incremental=False, rebuild_every=8,
        D0=None, callback=None, fractional=False):
    """Restricted closed-shell HF.  Converged when the RMS change of the
    density is below ``conv`` and its largest change below 100 ``conv``
    (electdiis's test, src/scf.f90:594).  With ``fractional`` the 2 ``nocc``
    electrons are spread over degenerate orbitals (aufbau_occupations): the
    spherically averaged atoms of the superposition-of-atomic-densities
    guess."""
    t_start = time.perf_counter()
    S, H = engine.overlap_core()
    enuc = engine.enuc()
    X = orthogonaliser(S)

    def diag(F):
        e, Cp = np.linalg.eigh(X.T @ F @ X)
        return e, X @ Cp

    def density(eps, C):
        if fractional:
            return (C * aufbau_occupations(eps, 2 * nocc)) @ C.T
        return _density(C, nocc)

    if D0 is None:
        eps, C = diag(H)
        D = density(eps, C)
    else:
        D = np.array(D0)
    fock_s = 0.0
    G = None
    D_built = None
    focks, errs = [], []
    history = []
    converged = False
    it = 0
    for it in range(1, max_iter + 1):
        t0 = time.perf_counter()
        if incremental and G is not None and (it - 1) % rebuild_every != 0:
            G = G + engine.fock2e(D - D_built)
        else:
            G = engine.fock2e(D)
        fock_s += time.perf_counter() - t0
        D_built = D
        F = H + G
        e_elec = 0.5 * float(np.sum(D * (H + F)))
        err = F @ D @ S - S @ D @ F
        err = X.T @ err @ X
        focks.append(F)
        errs.append(err)
        if len(focks) > diis_size:
            focks.pop(0)
            errs.pop(0)
        Fx = F
        if len(focks) > 1:
            m = len(focks)
            B = -np.ones((m + 1, m + 1))
            B[m, m] = 0.0
            for i in range(m):
                for j in range(i + 1):
                    B[i, j] = B[j, i] = float(np.sum(errs[i] * errs[j]))
            rhs = np.zeros(m + 1)
            rhs[m] = -1.0
            try:
                c = np.linalg.solve(B, rhs)[:m]
                Fx = sum(ci * Fi for ci, Fi in zip(c, focks))
            except np.linalg.LinAlgError:
                Fx = F
        eps, C = diag(Fx)
        D_new = density(eps, C)
        dD = D_new - D
        drms = float(np.sqrt(np.mean(dD * dD)))
        dmax = float(np.abs(dD).max())
        history.append((e_elec + enuc, drms, time.perf_counter() - t0))
        if callback:
            callback(it, e_elec + enuc, drms)
        D = D_new
        if drms < conv and dmax < 100.0 * conv:
            converged = True
            break
    # orbitals of the Fock matrix built from the final density's predecessor;
    # the energy is that of the last build (QUICK reports the same)
    eps, C = diag(F)
    return SCFResult(energy=e_elec + enuc, e_elec=e_elec, e_nuc=enuc, converged=converged, iterations=it,
                     D=D_built, C=C, eps=eps, nocc=nocc, history=history, fock_seconds=fock_s,
                     seconds=time.perf_counter() - t_start)


def sad_guess(mol, basis, atom_density):
    """Superposition of atomic densities (QUICK's default guess, getmolsad in
    src/getMolSad.f90): the block-diagonal density with each atom's block
    from ``atom_density(symbol)`` (nbf_atom x nbf_atom, the atom alone in the
    same basis), computed once per element."""
    D = np.zeros((basis.nbasis, basis.nbasis))
    cache = {}
    for i, sym in enumerate(mol.symbols):
        if sym not in cache:
            cache[sym] = atom_density(sym)
        f, l = basis.first_basis_function[i] - 1, basis.last_basis_function[i]
        D[f:l, f:l] = cache[sym]
    return D


class GpuEngine:
    """One-electron integrals, Fock build and gradients through this
    package's C ABI (``capi.Session``)."""

    def __init__(self, session, mol, basis, integral_cutoff=1e-10, prim_limit=1e-20, method=0, grad_cutoff=None):
        self.s = session
        self.mol = mol
        self.basis = basis
        self.cut = integral_cutoff
        self.plim = prim_limit
        self.method = method
        self.grad_cut = integral_cutoff if grad_cutoff is None else grad_cutoff
        self.nfock = 0

    def overlap_core(self):
        return self.s.oneint()

    def enuc(self):
        return self.mol.nuclear_repulsion()

    def fock2e(self, D):
        self.nfock += 1
        n = self.basis.nbasis
        return self.s.get2e(np.zeros((n, n), order="F"), D, shell_cut_matrix(self.basis, D), self.cut, self.plim,
                            self.method)

    def gradient(self, D, W):
        g = self.s.grad1e(D, W)
        return self.s.grad(g, D, shell_cut_matrix(self.basis, D), self.grad_cut, self.plim)


def gpu_atom_density(symbol, basis_name, device=0, conv=1e-7):
    """Spherically averaged atomic density on the GPU (fractional-occupation
    SCF of the atom alone); opens and closes its own session."""
    from .basis import build_basis
    from .capi import Session
    from .molecule import Molecule
    m = Molecule([symbol], np.zeros((1, 3)))
    b = build_basis(m.symbols, basis_name)
    s = Session(device)
    try:
        s.upload_molecule(m, b)
        r = rhf(GpuEngine(s, m, b, 1e-12, 1e-20), m.n_electrons / 2.0, conv=conv, max_iter=60, fractional=True)
    finally:
        s.close()
    return r.D


def run_rhf_gpu(mol, basis_name, integral_cutoff=1e-10, prim_limit=1e-20, conv=1e-8, gradient=False,
                mixed_cut=0.0, incremental=False, device=0, max_iter=100):
    """Energy (and gradient) of a closed-shell molecule on the GPU: the SAD
    guess, the DIIS SCF over the GPU Fock build, and the analytic gradient.
    Returns (SCFResult, gradient or None)."""
    from .basis import build_basis
    from .capi import Session
    b = build_basis(mol.symbols, basis_name)
    t0 = time.perf_counter()
    D0 = sad_guess(mol, b, lambda sym: gpu_atom_density(sym, basis_name, device))
    t_guess = time.perf_counter() - t0
    s = Session(device)
    try:
        s.upload_molecule(mol, b)
        if mixed_cut:
            s.set_mixed_precision(mixed_cut)
        eng = GpuEngine(s, mol, b, integral_cutoff, prim_limit)
        r = rhf(eng, mol.n_electrons // 2, conv=conv, D0=D0, incremental=incremental, max_iter=max_iter)
        g = eng.gradient(r.D, r.W) if gradient else None
    finally:
        s.close()
    r.seconds += t_guess
    return r, g
