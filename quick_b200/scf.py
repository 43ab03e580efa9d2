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


def rhf(engine, nocc, conv=1e-8, max_iter=100, diis_size=10, incremental=False, rebuild_every=8,
        D0=None, callback=None):
    """Restricted closed-shell HF.  Converged when the RMS change of the
    density is below ``conv`` and its largest change below 100 ``conv``
    (electdiis's test, src/scf.f90:594)."""
    t_start = time.perf_counter()
    S, H = engine.overlap_core()
    enuc = engine.enuc()
    X = orthogonaliser(S)

    def diag(F):
        e, Cp = np.linalg.eigh(X.T @ F @ X)
        return e, X @ Cp

    if D0 is None:
        eps, C = diag(H)
        D = _density(C, nocc)
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
        D_new = _density(C, nocc)
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
