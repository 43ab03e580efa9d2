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
    fock_builds: int = 0
    timings: dict = field(default_factory=dict)   # wall seconds per phase (run_rhf_device)
    graph_timings: dict = field(default_factory=dict)   # graph SCF: wall seconds of its steps

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
    xc = engine.xc if getattr(engine, "method", 0) else None

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
        if xc is not None:
            # Kohn-Sham: F = H + G(D; hybrid exchange) + V_xc, E = tr DH + tr DG / 2 + E_xc
            Vxc, Exc = xc(D)
            F = F + Vxc
            e_elec += Exc
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

    def xc(self, D):
        """(V_xc, E_xc) on QUICK's SG1 grid (gpu_getxc_)."""
        from .basis import sigrad2
        if not hasattr(self, "_sg"):
            self._sg = sigrad2(self.basis)
        n = self.basis.nbasis
        V, exc, _, _ = self.s.getxc(np.zeros((n, n), order="F"), D, self._sg, method=self.method)
        return V, exc

    def gradient(self, D, W):
        g = self.s.grad1e(D, W)
        return self.s.grad(g, D, shell_cut_matrix(self.basis, D), self.grad_cut, self.plim)


def gpu_atom_density(symbol, basis_name, device=0, conv=1e-7, session=None):
    """Spherically averaged atomic density on the GPU (fractional-occupation
    SCF of the atom alone), in ``session`` if given (the atom replaces what
    was uploaded), else in a session of its own."""
    from .basis import build_basis
    from .capi import Session
    from .molecule import Molecule
    m = Molecule([symbol], np.zeros((1, 3)))
    b = build_basis(m.symbols, basis_name)
    s = Session(device) if session is None else session
    try:
        s.upload_molecule(m, b)
        r = rhf(GpuEngine(s, m, b, 1e-12, 1e-20), m.n_electrons / 2.0, conv=conv, max_iter=60, fractional=True)
    finally:
        if session is None:
            s.close()
    return r.D


def run_rhf_gpu(mol, basis_name, integral_cutoff=1e-10, prim_limit=1e-20, conv=1e-8, gradient=False,
                mixed_cut=0.0, incremental=False, device=0, max_iter=100, method=0):
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
        eng = GpuEngine(s, mol, b, integral_cutoff, prim_limit, method=method)
        r = rhf(eng, mol.n_electrons // 2, conv=conv, D0=D0, incremental=incremental, max_iter=max_iter)
        g = eng.gradient(r.D, r.W) if gradient else None
    finally:
        s.close()
    r.seconds += t_guess
    return r, g


class DeviceRHF:
    """The SCF with every matrix resident on the GPU.

    The one-electron integrals (qb_oneint_device), the density screen
    (qb_upload_cutoff_device), the Fock build (qb_fock_device) and the
    gradients (qb_grad1e_device, qb_grad_device) run through the library's
    device entry points on the caller's stream; the dense linear algebra of
    the SCF (orthogonalisation, DIIS, diagonalisation by cuSOLVER) uses torch
    tensors on the same stream.  Per iteration only the DIIS overlaps and the
    convergence scalars come back to the host."""

    def __init__(self, session, mol, basis, integral_cutoff=1e-10, prim_limit=1e-20, grad_cutoff=None, method=0,
                 xc_grid=1):
        import ctypes as C

        import torch

        from . import capi
        self.torch, self.C, self.capi = torch, C, capi
        self.lib = capi.lib()
        self.s, self.mol, self.basis = session, mol, basis
        self.cut, self.plim = integral_cutoff, prim_limit
        self.grad_cut = integral_cutoff if grad_cutoff is None else grad_cutoff
        # a stream of our own: the library treats a null stream as "use the
        # library's stream", so torch's legacy default stream cannot be shared
        self.stream = torch.cuda.Stream()
        self.lib.qb_set_stream(C.c_void_p(self.stream.cuda_stream))
        n = basis.nbasis
        self.opts = dict(dtype=torch.float64, device=torch.device("cuda", torch.cuda.current_device()))
        with torch.cuda.stream(self.stream):
            self.S = torch.empty((n, n), **self.opts)
            self.H = torch.empty((n, n), **self.opts)
            self._rc(self.lib.qb_oneint_device(self._p(self.S), self._p(self.H)))
        self.nfock = 0
        # 0 HF, 1 B3LYP, 2 BLYP: the exchange fraction of the Fock build and the functional
        self.method = method
        self.lib.gpu_upload_method_(C.byref(C.c_int(method)))
        if method:
            from .basis import sigrad2
            self.sg = np.ascontiguousarray(sigrad2(basis))
            # 1: QUICK's SG1 grid, 2: 75 x 302 points per atom with Becke's partition
            self._rc(self.lib.qb_set_xc_grid(C.c_int(xc_grid)))

    def xc(self, D):
        """(V_xc symmetrised, E_xc) for the device density D (qb_xc_device)."""
        torch, C = self.torch, self.C
        V = torch.zeros_like(D)
        exc, na = C.c_double(0.0), C.c_double(0.0)
        self._rc(self.lib.qb_xc_device(self._p(D), self.sg.ctypes.data_as(C.c_void_p), self._p(V), C.byref(exc),
                                       C.byref(na)))
        # the library fills V(j, i), j >= i of the column-major matrix: the upper triangle of this view
        V = torch.triu(V) + torch.triu(V, 1).T
        return V, exc.value

    def _p(self, t):
        return self.C.c_void_p(t.data_ptr())

    def _rc(self, rc):
        if rc:
            self.capi.check()
            raise self.capi.QuickB200Error(rc, "device SCF call failed")

    def fock(self, Dd, Oin):
        """Oin + G(Dd), density screen from Dd."""
        F = self.torch.empty_like(Oin)
        C = self.C
        self._rc(self.lib.qb_upload_cutoff_device(self._p(Dd), C.c_double(self.cut), C.c_double(self.plim)))
        self._rc(self.lib.qb_fock_device(self._p(Dd), self._p(Oin), self._p(F)))
        self.nfock += 1
        return F

    def fock_into(self, Dd, Oin, Out):
        """Out = Oin + G(Dd) with the density screen from Dd (Out may be Oin)."""
        C = self.C
        self._rc(self.lib.qb_upload_cutoff_device(self._p(Dd), C.c_double(self.cut), C.c_double(self.plim)))
        self._rc(self.lib.qb_fock_device(self._p(Dd), self._p(Oin), self._p(Out)))
        self.nfock += 1

    def run(self, nocc, D0, conv=1e-8, max_iter=100, diis_size=10, incremental=False, rebuild_every=8,
            graph=False, sp2_iters=48):
        """graph=True: every iteration after the first is one CUDA-graph replay
        (Hartree-Fock only; see _run_graph)."""
        with self.torch.cuda.stream(self.stream):
            if graph:
                if self.method:
                    raise ValueError("the graph-captured SCF is Hartree-Fock only (the XC quadrature captures "
                                     "its own graph)")
                return self._run_graph(nocc, D0, conv, max_iter, min(diis_size, 32), incremental, rebuild_every,
                                       sp2_iters)
            return self._run(nocc, D0, conv, max_iter, diis_size, incremental, rebuild_every)

    def _sp2(self, Fo, nocc, iters):
        """Projector onto the nocc lowest eigenvectors of the symmetric Fo by
        Niklasson's second-order spectral projection (SP2, Phys. Rev. B 66,
        155115 (2002)): X0 = (e_max - Fo)/(e_max - e_min) with Gershgorin
        bounds, then X <- X^2 when tr X > nocc, else X <- 2X - X^2.  Matrix
        products and a device-side choice only, so it can be captured."""
        torch = self.torch
        d = Fo.diagonal()
        r = Fo.abs().sum(1) - d.abs()
        emin, emax = (d - r).min(), (d + r).max()
        eye = torch.eye(Fo.shape[0], **self.opts)
        X = (emax * eye - Fo) / (emax - emin)
        for _ in range(iters):
            X2 = X @ X
            X = torch.where(X.diagonal().sum() > nocc, X2, 2.0 * X - X2)
        return X

    def _run_graph(self, nocc, D0, conv, max_iter, M, incremental, rebuild_every, sp2_iters):
        """The SCF with each iteration captured as a CUDA graph and replayed:
        density screen and Fock build (full, or incremental F + G(D - D_built)
        with a full rebuild every rebuild_every iterations: one graph each),
        the DIIS error X^T (F D S - S D F) X into a ring of M slots, the
        overlaps of all slots by one GEMM, the Pulay coefficients on the device
        (qb_diis_solve_device), the extrapolated Fock matrix, and the new
        density from SP2 purification (_sp2) in place of a diagonalisation.
        The host reads three scalars per iteration (energy, RMS and largest
        density change) for QUICK's convergence test; the eigenvectors are
        formed once, after convergence."""
        torch = self.torch
        t_start = time.perf_counter()
        S, H = self.S, self.H
        s, U = torch.linalg.eigh(S)
        keep = s > 1e-4
        X = U[:, keep] * s[keep].rsqrt()
        if bool(keep.all()):
            X = X @ U.T
        Xt = X.T.contiguous()
        n = S.shape[0]
        m = X.shape[1]
        opts = self.opts
        gt = {"orthogonaliser": time.perf_counter() - t_start}
        D = torch.as_tensor(np.ascontiguousarray(D0), **opts).clone()
        D_built = torch.zeros_like(D)
        dIn = torch.zeros_like(D)
        F2 = torch.zeros_like(D)
        focks = torch.zeros((M, n, n), **opts)
        errs = torch.zeros((M, m, m), **opts)
        it_dev = torch.zeros((), dtype=torch.int64, device=D.device)
        slot = torch.zeros((), dtype=torch.int64, device=D.device)
        cvec = torch.zeros(M, **opts)
        ar = torch.arange(M, device=D.device)
        stats = torch.zeros(3, **opts)
        enuc = self.mol.nuclear_repulsion()
        lib, C = self.lib, self.C

        def step(incr):
            if incr:
                torch.sub(D, D_built, out=dIn)
                self.fock_into(dIn, F2, F2)
            else:
                self.fock_into(D, H, F2)
            D_built.copy_(D)
            e = 0.5 * (D * (H + F2)).sum()
            FDS = F2 @ D @ S
            err = Xt @ (FDS - FDS.T) @ X
            torch.remainder(it_dev, M, out=slot)
            focks.index_copy_(0, slot.view(1), F2.unsqueeze(0))
            errs.index_copy_(0, slot.view(1), err.unsqueeze(0))
            E = errs.view(M, -1)
            B = (E @ E.T).contiguous()
            w = (ar <= it_dev).to(torch.float64)
            self._rc(lib.qb_diis_solve_device(self._p(B), self._p(w), C.c_int(M), self._p(slot), self._p(cvec)))
            Fx = (cvec.view(M, 1, 1) * focks).sum(0)
            P = self._sp2(Xt @ Fx @ X, nocc, sp2_iters)
            Dn = 2.0 * (X @ P @ Xt)
            dD = Dn - D
            stats.copy_(torch.stack([e, dD.square().mean().sqrt(), dD.abs().max()]))
            D.copy_(Dn)
            it_dev.add_(1)

        history = []
        converged = False
        it = 1
        # iteration 1 eagerly (it also warms up the library, cuBLAS and the allocator)
        t0 = time.perf_counter()
        step(False)
        vals = stats.cpu().numpy()
        history.append((float(vals[0]) + enuc, float(vals[1]), time.perf_counter() - t0))
        if vals[1] < conv and vals[2] < 100.0 * conv:
            converged = True
        graphs = {}
        if not converged:
            torch.cuda.synchronize()
            t_cap = time.perf_counter()
            for incr in ((False, True) if incremental else (False,)):
                g = torch.cuda.CUDAGraph()
                pool = graphs[False].pool() if graphs else None
                with torch.cuda.graph(g, stream=self.stream, pool=pool):
                    step(incr)
                self.nfock -= 1          # captured, not built
                graphs[incr] = g
            gt["capture"] = time.perf_counter() - t_cap
            for it in range(2, max_iter + 1):
                t0 = time.perf_counter()
                graphs[incremental and (it - 1) % rebuild_every != 0].replay()
                self.nfock += 1
                vals = stats.cpu().numpy()
                history.append((float(vals[0]) + enuc, float(vals[1]), time.perf_counter() - t0))
                if vals[1] < conv and vals[2] < 100.0 * conv:
                    converged = True
                    break
        e_elec = float(vals[0])
        t_fin = time.perf_counter()
        eps, Cp = torch.linalg.eigh(Xt @ F2 @ X)
        Cm = X @ Cp
        self.D_dev, self.C_dev, self.eps_dev = D_built.clone(), Cm, eps
        torch.cuda.synchronize()
        gt["final_eigh"] = time.perf_counter() - t_fin
        t_rel = time.perf_counter()
        graphs.clear()
        gt["release"] = time.perf_counter() - t_rel
        res = SCFResult(energy=e_elec + enuc, e_elec=e_elec, e_nuc=enuc, converged=converged, iterations=it,
                        D=D_built.cpu().numpy(), C=Cm.cpu().numpy(), eps=eps.cpu().numpy(), nocc=nocc,
                        history=history, seconds=time.perf_counter() - t_start)
        res.graph_timings = {k: round(v, 4) for k, v in gt.items()}
        return res

    def _run(self, nocc, D0, conv, max_iter, diis_size, incremental, rebuild_every):
        torch = self.torch
        t_start = time.perf_counter()
        S, H = self.S, self.H
        s, U = torch.linalg.eigh(S)
        keep = s > 1e-4
        X = U[:, keep] * s[keep].rsqrt()
        if bool(keep.all()):
            X = X @ U.T
        D = torch.as_tensor(np.ascontiguousarray(D0), **self.opts)
        enuc = self.mol.nuclear_repulsion()
        focks, errs = [], []
        B = np.zeros((0, 0))
        history = []
        converged = False
        F = F2 = D_built = None
        e_elec = 0.0
        it = 0
        for it in range(1, max_iter + 1):
            t0 = time.perf_counter()
            if incremental and F2 is not None and (it - 1) % rebuild_every != 0:
                F2 = self.fock(D - D_built, F2)
            else:
                F2 = self.fock(D, H)
            D_built = D
            e_t = 0.5 * (D * (H + F2)).sum()
            F = F2
            if self.method:
                Vxc, Exc = self.xc(D)
                F = F2 + Vxc
                e_t = e_t + Exc
            FDS = F @ D @ S
            err = X.T @ (FDS - FDS.T) @ X
            focks.append(F)
            errs.append(err)
            if len(focks) > diis_size:
                focks.pop(0)
                errs.pop(0)
                B = B[1:, 1:]
            row = torch.stack([(e * err).sum() for e in errs]).cpu().numpy()
            m = len(errs)
            Bn = np.zeros((m, m))
            Bn[:m - 1, :m - 1] = B
            Bn[m - 1, :] = row
            Bn[:, m - 1] = row
            B = Bn
            Fx = F
            if m > 1:
                A = -np.ones((m + 1, m + 1))
                A[m, m] = 0.0
                A[:m, :m] = B
                rhs = np.zeros(m + 1)
                rhs[m] = -1.0
                try:
                    c = np.linalg.solve(A, rhs)[:m]
                    Fx = sum(float(ci) * Fi for ci, Fi in zip(c, focks))
                except np.linalg.LinAlgError:
                    Fx = F
            eps, Cp = torch.linalg.eigh(X.T @ Fx @ X)
            Co = (X @ Cp)[:, :nocc]
            D_new = 2.0 * Co @ Co.T
            dD = D_new - D
            vals = torch.stack([e_t, dD.square().mean().sqrt(), dD.abs().max()]).cpu().numpy()
            e_elec, drms, dmax = float(vals[0]), float(vals[1]), float(vals[2])
            history.append((e_elec + enuc, drms, time.perf_counter() - t0))
            D = D_new
            if drms < conv and dmax < 100.0 * conv:
                converged = True
                break
        eps, Cp = torch.linalg.eigh(X.T @ F @ X)
        Cm = X @ Cp
        self.D_dev, self.C_dev, self.eps_dev = D_built, Cm, eps
        torch.cuda.synchronize()
        return SCFResult(energy=e_elec + enuc, e_elec=e_elec, e_nuc=enuc, converged=converged, iterations=it,
                         D=D_built.cpu().numpy(), C=Cm.cpu().numpy(), eps=eps.cpu().numpy(), nocc=nocc,
                         history=history, seconds=time.perf_counter() - t_start)

    def gradient(self):
        """Full nuclear gradient (3 natom) at the last SCF's density."""
        with self.torch.cuda.stream(self.stream):
            return self._gradient()

    def _gradient(self):
        torch, C = self.torch, self.C
        nocc = self.mol.n_electrons // 2
        Co = self.C_dev[:, :nocc]
        W = 2.0 * (Co * self.eps_dev[:nocc]) @ Co.T
        D = self.D_dev
        g = torch.zeros(3 * self.mol.natom, **self.opts)
        self._rc(self.lib.qb_grad1e_device(self._p(D), self._p(W), self._p(g)))
        self._rc(self.lib.qb_upload_cutoff_device(self._p(D), C.c_double(self.grad_cut), C.c_double(self.plim)))
        self._rc(self.lib.qb_grad_device(self._p(D), self._p(g)))
        if self.method:
            # the exchange-correlation term (the two-electron one above carries the exchange fraction)
            self._rc(self.lib.qb_xc_grad_device(self._p(D), self.sg.ctypes.data_as(C.c_void_p), self._p(g)))
        return g.cpu().numpy()


_ATOM_DENSITY = {}


def run_rhf_device(mol, basis_name, integral_cutoff=1e-10, prim_limit=1e-20, conv=1e-8, gradient=True,
                   mixed_cut=0.0, incremental=False, device=0, max_iter=100, method=0, session=None, graph=False,
                   xc_grid=1):
    """Energy and gradient with the device-resident SCF (DeviceRHF) from the
    SAD guess; atomic densities are cached per (element, basis).  Returns
    (SCFResult, gradient or None); SCFResult.seconds covers guess, set-up,
    SCF and gradient (timings holds each, and the session close apart).  ``session``: an open capi.Session to upload into and keep
    open (molecule after molecule without re-initialising the library); by
    default a session is opened and closed around the call.  graph=True: each
    SCF iteration after the first is one CUDA-graph replay (DeviceRHF.run).
    method 1 / 2 (B3LYP / BLYP): Kohn-Sham, with the XC term in the gradient;
    xc_grid 1 = QUICK's SG1 grid, 2 = the 75 x 302 Becke grid."""
    from .basis import build_basis
    from .capi import Session
    t0 = time.perf_counter()
    b = build_basis(mol.symbols, basis_name)

    def atom(sym):
        key = (sym, basis_name)
        if key not in _ATOM_DENSITY:
            _ATOM_DENSITY[key] = gpu_atom_density(sym, basis_name, device, session=session)
        return _ATOM_DENSITY[key]

    D0 = sad_guess(mol, b, atom)
    t1 = time.perf_counter()
    own = session is None
    s = Session(device) if own else session
    try:
        s.upload_molecule(mol, b)
        t_up = time.perf_counter()
        s.set_mixed_precision(mixed_cut)
        eng = DeviceRHF(s, mol, b, integral_cutoff, prim_limit, method=method, xc_grid=xc_grid)
        eng.torch.cuda.synchronize()
        t2 = time.perf_counter()
        r = eng.run(mol.n_electrons // 2, D0, conv=conv, incremental=incremental, max_iter=max_iter, graph=graph)
        t3 = time.perf_counter()
        g = eng.gradient() if gradient else None
        t4 = time.perf_counter()
        r.fock_builds = eng.nfock
    finally:
        t5 = time.perf_counter()
        if own:
            s.close()
        else:
            # the engine's stream dies with it: hand the session back its own
            from .capi import lib
            lib().qb_set_stream(None)
    # the work of one molecule; closing the session (freeing the library's
    # device memory, which a long-lived session does once) is reported apart
    r.seconds = t4 - t0
    r.timings = dict(guess=t1 - t0, setup=t2 - t1, scf=t3 - t2, gradient=t4 - t3, close=time.perf_counter() - t5,
                     setup_upload=t_up - t1)
    return r, g


def run_batch_rhf(mols, basis_name, integral_cutoff=1e-10, prim_limit=1e-20, conv=1e-8, max_iter=100, diis_size=8,
                  mixed_cut=0.0, incremental=True, rebuild_every=8, gradient=True, device=0, session=None,
                  sp2_iters=48):
    """Closed-shell SCF (and gradient) of many molecules advanced together:
    every iteration is one batched Fock build for all of them
    (qb_batch_fock_device: one screen launch and one launch per angular class)
    and batched dense algebra on zero-padded blocks (torch bmm): DIIS per
    molecule, and the new density by SP2 purification (DeviceRHF._sp2's
    scheme, with each padding diagonal set to the block's upper spectral bound
    so it stays unoccupied).  With incremental=True the builds take
    D - D_built (full rebuild every rebuild_every iterations), so molecules
    that have converged add no quartets.  The two-electron gradient is one
    batched call (qb_batch_grad_device); the one-electron gradient runs per
    molecule.  Returns (list of SCFResult, list of gradients or None, timings)."""
    import ctypes as C

    import torch

    from .basis import build_basis
    from .capi import QuickB200Error, Session, check, lib

    L = lib()
    t0 = time.perf_counter()
    own = session is None
    s = Session(device) if own else session
    dev = torch.device("cuda", torch.cuda.current_device())
    opts = dict(dtype=torch.float64, device=dev)
    stream = torch.cuda.Stream()
    L.qb_set_stream(C.c_void_p(stream.cuda_stream))
    p = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731

    def rc(v):
        if v:
            check()
            raise QuickB200Error(v, "batched SCF call failed")

    timings = {}
    try:
        with torch.cuda.stream(stream):
            nmol = len(mols)
            bases = [build_basis(m.symbols, basis_name) for m in mols]
            ns = [b.nbasis for b in bases]
            nmax = max(ns)
            nocc = torch.tensor([m.n_electrons // 2 for m in mols], **opts)
            S = torch.zeros((nmol, nmax, nmax), **opts)
            H = torch.zeros((nmol, nmax, nmax), **opts)
            D = torch.zeros((nmol, nmax, nmax), **opts)
            rc(L.qb_batch_reset())

            def atom(sym):
                key = (sym, basis_name)
                if key not in _ATOM_DENSITY:
                    _ATOM_DENSITY[key] = gpu_atom_density(sym, basis_name, device, session=s)
                return _ATOM_DENSITY[key]

            for i, (m, b) in enumerate(zip(mols, bases)):
                n = b.nbasis
                s.upload_molecule(m, b)
                rc(L.qb_batch_add())
                Si = torch.empty((n, n), **opts)
                Hi = torch.empty((n, n), **opts)
                rc(L.qb_oneint_device(p(Si), p(Hi)))
                S[i, :n, :n] = Si
                H[i, :n, :n] = Hi
                D[i, :n, :n] = torch.as_tensor(np.ascontiguousarray(sad_guess(m, b, atom)), **opts)
            s.set_mixed_precision(mixed_cut)
            rc(L.qb_batch_finalize(C.c_double(integral_cutoff), C.c_double(prim_limit)))
            nb_ = np.zeros(nmol, dtype=np.int32)
            na_ = np.zeros(nmol, dtype=np.int32)
            off = np.zeros(nmol, dtype=np.int64)
            L.qb_batch_layout(nb_.ctypes.data_as(C.c_void_p), na_.ctypes.data_as(C.c_void_p),
                              off.ctypes.data_as(C.c_void_p), C.c_int(nmol))
            # packed element e = a + b n_i of molecule i <-> padded [i, b, a] (symmetric blocks)
            idx = np.concatenate([i * nmax * nmax + (np.arange(n)[None, :] * nmax + np.arange(n)[:, None]).T.ravel()
                                  for i, n in enumerate(ns)])
            pidx = torch.as_tensor(idx, device=dev)
            ntot_pk = int(off[-1] + ns[-1] * ns[-1])

            def pack(X):
                return X.reshape(-1).index_select(0, pidx).contiguous()

            def unpack(x):
                X = torch.zeros((nmol, nmax, nmax), **opts)
                X.view(-1).index_copy_(0, pidx, x)
                return X

            real = torch.zeros((nmol, nmax), dtype=torch.bool, device=dev)
            for i, n in enumerate(ns):
                real[i, :n] = True
            pad = (~real).to(torch.float64)
            # Cholesky orthogonalisers X = L^-T (S = L L^T, X^T S X = 1),
            # identity on the padding: one batched factorisation and
            # triangular solve instead of a batched eigh (0.8 s for 256
            # molecules); the converged densities do not depend on the
            # choice.  A pivot L_ii^2 bounds the smallest eigenvalue of S from
            # above, so a pivot below 1e-4 means a near-linear dependence,
            # which this driver does not remove (run_rhf_device does).
            Sid = S + torch.diag_embed(pad)
            Lc, info = torch.linalg.cholesky_ex(Sid)
            if bool((info != 0).any()) or bool((Lc.diagonal(dim1=1, dim2=2).square() < 1e-4).any()):
                raise QuickB200Error(1, "run_batch_rhf: the overlap is near-singular (use run_rhf_device)")
            eye = torch.eye(nmax, **opts).expand(nmol, nmax, nmax)
            Xt = torch.linalg.solve_triangular(Lc, eye, upper=False).contiguous()
            X = Xt.transpose(1, 2)
            Hp = pack(H)
            enuc = torch.tensor([m.nuclear_repulsion() for m in mols], **opts)
            nel = torch.tensor(ns, **opts) ** 2
            torch.cuda.synchronize()
            t1 = time.perf_counter()
            timings["setup"] = t1 - t0
            M = diis_size
            focks = torch.zeros((M, nmol, nmax, nmax), **opts)
            errs = torch.zeros((M, nmol, nmax, nmax), **opts)
            F2p = torch.zeros(ntot_pk, **opts)
            Dbuilt = torch.zeros(ntot_pk, **opts)
            converged = torch.zeros(nmol, dtype=torch.bool, device=dev)
            iters = torch.zeros(nmol, dtype=torch.int64, device=dev)
            e_t = torch.zeros(nmol, **opts)
            it = 0
            for it in range(1, max_iter + 1):
                Dp = pack(D)
                if incremental and it > 1 and (it - 1) % rebuild_every != 0:
                    dDp = Dp - Dbuilt
                    rc(L.qb_batch_fock_device(p(dDp), p(F2p), p(F2p)))
                else:
                    rc(L.qb_batch_fock_device(p(Dp), p(Hp), p(F2p)))
                Dbuilt = Dp
                F = unpack(F2p)
                e_t = 0.5 * (D * (H + F)).sum(dim=(1, 2))
                FDS = F @ D @ S
                err = Xt @ (FDS - FDS.transpose(1, 2)) @ X
                slot = (it - 1) % M
                focks[slot] = F
                errs[slot] = err
                m_ = min(it, M)
                E = errs[:m_].permute(1, 0, 2, 3).reshape(nmol, m_, -1)
                B = E @ E.transpose(1, 2)
                A = -torch.ones((nmol, m_ + 1, m_ + 1), **opts)
                A[:, m_, m_] = 0.0
                A[:, :m_, :m_] = B
                rhs = torch.zeros((nmol, m_ + 1), **opts)
                rhs[:, m_] = -1.0
                c, info = torch.linalg.solve_ex(A, rhs)
                c = torch.where((info == 0)[:, None], c[:, :m_],
                                torch.nn.functional.one_hot(torch.tensor(slot, device=dev), m_).to(torch.float64))
                Fx = torch.einsum("nm,mnij->nij", c, focks[:m_])
                Fo = Xt @ Fx @ X
                # SP2 with the padding parked at the block's upper bound (projector value 0 there)
                d = Fo.diagonal(dim1=1, dim2=2)
                r = Fo.abs().sum(2) - d.abs()
                emin = torch.where(real, d - r, torch.full_like(d, 1e300)).min(1).values
                emax = torch.where(real, d + r, torch.full_like(d, -1e300)).max(1).values
                Fo = Fo + torch.diag_embed(pad * emax[:, None])
                eye = torch.eye(nmax, **opts).expand(nmol, nmax, nmax)
                P = (emax[:, None, None] * eye - Fo) / (emax - emin)[:, None, None]
                for _ in range(sp2_iters):
                    P2 = P @ P
                    tr = P.diagonal(dim1=1, dim2=2).sum(1)
                    P = torch.where((tr > nocc)[:, None, None], P2, 2.0 * P - P2)
                Dn = 2.0 * (X @ P @ Xt)
                dD = Dn - D
                drms = (dD.square().sum(dim=(1, 2)) / nel).sqrt()
                dmax = dD.abs().amax(dim=(1, 2))
                done = (drms < conv) & (dmax < 100.0 * conv)
                iters = torch.where(converged, iters, torch.full_like(iters, it))
                converged = converged | done
                # a converged molecule keeps the density of its last build (its energy's)
                D = torch.where(converged[:, None, None], D, Dn)
                if bool(converged.all()):
                    break
            torch.cuda.synchronize()
            t2 = time.perf_counter()
            timings["scf"] = t2 - t1
            energy = (e_t + enuc).cpu().numpy()
            # D is the density of the last build for converged molecules
            Dfin = unpack(Dbuilt)
            grads = None
            if gradient:
                g2 = torch.zeros(3 * int(na_.sum()), **opts)
                rc(L.qb_batch_grad_device(p(Dbuilt), p(g2)))
                # W = 2 sum_occ e_k C_k C_k^T = D F D / 2 for the converged
                # closed-shell density (D = 2 C_occ C_occ^T, F C = S C e):
                # two batched products instead of a batched eigh
                W = 0.5 * (Dfin @ F @ Dfin)
                # one-electron terms per molecule into one device vector (the
                # molecules' atoms in order, like g2), read back once
                g1 = torch.zeros_like(g2)
                a0 = 0
                for i, (m, b) in enumerate(zip(mols, bases)):
                    n = b.nbasis
                    s.upload_molecule(m, b, pairs=False)
                    Di = Dfin[i, :n, :n].contiguous()
                    Wi = W[i, :n, :n].contiguous()
                    rc(L.qb_grad1e_device(p(Di), p(Wi), p(g1[3 * a0:3 * (a0 + m.natom)])))
                    a0 += m.natom
                gh = (g1 + g2).cpu().numpy()
                grads = []
                a0 = 0
                for m in mols:
                    grads.append(gh[3 * a0:3 * (a0 + m.natom)].copy())
                    a0 += m.natom
            torch.cuda.synchronize()
            timings["gradient"] = time.perf_counter() - t2
            conv_h = converged.cpu().numpy()
            it_h = iters.cpu().numpy()
            Dh = Dfin.cpu().numpy()
            results = [SCFResult(energy=float(energy[i]), e_elec=float(energy[i] - enuc[i]), e_nuc=float(enuc[i]),
                                 converged=bool(conv_h[i]), iterations=int(it_h[i]),
                                 D=Dh[i, :ns[i], :ns[i]], C=None, eps=None, nocc=mols[i].n_electrons // 2,
                                 history=[], seconds=0.0) for i in range(nmol)]
    finally:
        L.qb_batch_reset()
        L.qb_set_stream(None)
        if own:
            s.close()
    timings["total"] = time.perf_counter() - t0
    return results, grads, timings
