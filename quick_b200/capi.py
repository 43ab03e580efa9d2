"""ctypes binding of ``libquickb200.so`` (the C ABI in include/quick_b200.h).

The call sequence mirrors QUICK's Fortran host: ``upload_molecule`` is the
start-up part of src/main.f90:84-177, ``get2e`` one Fock build of
src/hfoperator.f90:76-98.  Every call checks the bridge's sticky status and
raises ``QuickB200Error`` with its message; there is no fallback path.
"""
import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libquickb200.so")

_P = C.c_void_p


class QuickB200Error(RuntimeError):
    pass


_lib = None


def lib():
    """Load the CUDA library; raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise QuickB200Error("libquickb200.so not built: run `python -m quick_b200.build` "
                                 "(expected at %s)" % LIB_PATH)
        _lib = C.CDLL(LIB_PATH)
        _lib.qb_last_error.restype = C.c_char_p
    return _lib


def _ptr(a):
    return a.ctypes.data_as(_P)


def _i(v):
    return C.byref(C.c_int(int(v)))


def _d(v):
    return C.byref(C.c_double(float(v)))


def check():
    r = lib()
    st = r.qb_status()
    if st:
        msg = r.qb_last_error().decode()
        r.qb_clear_error()
        raise QuickB200Error("quick_b200 error %d: %s" % (st, msg))


class Session:
    """One molecule resident on the GPU behind QUICK's gpu_* entry points."""

    def __init__(self, device=0):
        r = lib()
        r.qb_clear_error()
        r.gpu_startup_()
        r.gpu_set_device_(_i(device))
        r.gpu_init_()
        check()
        self._keep = []
        self.nbasis = 0

    def _arr(self, a, dt):
        x = np.asfortranarray(a, dtype=dt)
        self._keep.append(x)
        return _ptr(x)

    def upload_molecule(self, mol, basis, YCutoff=None, cutPrim=None, pairs=True):
        """Start-up uploads; YCutoff / cutPrim default to the GPU Schwarz kernel.
        pairs=False: coordinates, charges and basis only (enough for the
        one-electron integrals and gradient), no Schwarz bounds or pair list."""
        r = lib()
        b = basis
        self.basis = b
        self.nbasis = b.nbasis
        self.nshell = b.nshell
        I32, F64 = np.int32, np.float64
        r.gpu_setup_(_i(mol.natom), _i(b.nbasis), _i(mol.n_electrons), _i(mol.mult), _i(mol.charge),
                     _i(len(set(mol.symbols))))
        r.gpu_upload_xyz_(self._arr(mol.xyz_bohr, F64))
        r.gpu_upload_atom_and_chg_(self._arr(mol.atomic_numbers, I32),
                                   self._arr(mol.atomic_numbers.astype(F64), F64))
        r.gpu_upload_basis_(_i(b.nshell), _i(b.nprim), _i(b.jshell), _i(b.jbasis), _i(b.maxcontract),
                            self._arr(b.ncontract, I32), self._arr(b.itype, I32), self._arr(b.aexp, F64),
                            self._arr(b.dcoeff, F64), self._arr(b.first_basis_function, I32),
                            self._arr(b.last_basis_function, I32), self._arr(b.first_shell_basis_function, I32),
                            self._arr(b.last_shell_basis_function, I32), self._arr(b.ncenter, I32),
                            self._arr(b.kstart, I32), self._arr(b.katom, I32), self._arr(b.ktype, I32),
                            self._arr(b.kprim, I32), self._arr(b.kshell, I32), self._arr(b.Ksumtype, I32),
                            self._arr(b.Qnumber, I32), self._arr(b.Qstart, I32), self._arr(b.Qfinal, I32),
                            self._arr(b.Qsbasis, I32), self._arr(b.Qfbasis, I32), self._arr(b.gccoeff, F64),
                            self._arr(b.cons, F64), self._arr(b.gcexpo, F64), self._arr(b.KLMN, I32))
        check()
        if not pairs:
            return
        if YCutoff is None:
            YCutoff, cutPrim = self.schwarz()
        r.gpu_upload_cutoff_matrix_(self._arr(YCutoff, F64), self._arr(cutPrim, F64))
        check()
        self.YCutoff, self.cutPrim = YCutoff, cutPrim

    def schwarz(self):
        b = self.basis
        Y = np.zeros((b.nshell, b.nshell), order="F")
        cp = np.zeros((b.jbasis, b.jbasis), order="F")
        lib().gpu_schwarz_(_ptr(Y), _ptr(cp))
        check()
        return Y, cp

    def get2e(self, O, dense, cutMatrix, integral_cutoff, prim_limit, method=0):
        """O + G(dense): QUICK's upload_method / calculated / cutoff + gpu_get2e_."""
        r = lib()
        n = self.nbasis
        o = np.array(O, order="F", dtype=np.float64)
        co = np.zeros((1,), dtype=np.float64)
        d = np.asfortranarray(dense, dtype=np.float64)
        cm = np.asfortranarray(cutMatrix, dtype=np.float64)
        r.gpu_upload_method_(_i(method))
        r.gpu_upload_calculated_(_ptr(o), _ptr(co), _ptr(co), _ptr(d))
        r.gpu_upload_cutoff_(_ptr(cm), _d(integral_cutoff), _d(prim_limit), None)
        r.gpu_get2e_(_ptr(o))
        check()
        return o

    def grad(self, grad_in, dense, cutMatrix, integral_cutoff, prim_limit, grad_cutoff=1e-7):
        """grad_in + dE2/dR: QUICK's upload_calculated / cutoff / grad + gpu_grad_
        (src/gradient.f90:279-286).  grad_in is QUICK's (3, natom) gradient."""
        r = lib()
        n = self.nbasis
        o = np.zeros((n, n), order="F")
        co = np.zeros((1,), dtype=np.float64)
        d = np.asfortranarray(dense, dtype=np.float64)
        cm = np.asfortranarray(cutMatrix, dtype=np.float64)
        g = np.array(grad_in, dtype=np.float64).ravel(order="F").copy()
        r.gpu_upload_calculated_(_ptr(o), _ptr(co), _ptr(co), _ptr(d))
        r.gpu_upload_cutoff_(_ptr(cm), _d(integral_cutoff), _d(prim_limit), None)
        r.gpu_upload_grad_(_ptr(g), _d(grad_cutoff))
        r.gpu_grad_(_ptr(g))
        check()
        return g

    def aoint(self, path, least_cutoff, max_cutoff):
        """QUICK's gpu_aoint_: the unique integrals into the file at path;
        returns how many were written."""
        r = lib()
        num = C.c_int(0)
        name = (path + " ").encode()
        r.gpu_aoint_(C.byref(C.c_double(least_cutoff)), C.byref(C.c_double(max_cutoff)), C.byref(num),
                     C.c_char_p(name))
        check()
        return num.value

    def addint(self, O, dense, path, nint, method=0):
        """QUICK's gpu_upload_method_ / gpu_upload_calculated_ + gpu_addint_:
        O + G(dense) from the stored integrals."""
        r = lib()
        o = np.array(O, order="F", dtype=np.float64)
        co = np.zeros((1,), dtype=np.float64)
        d = np.asfortranarray(dense, dtype=np.float64)
        r.gpu_upload_method_(_i(method))
        r.gpu_upload_calculated_(_ptr(o), _ptr(co), _ptr(co), _ptr(d))
        r.gpu_addint_(_ptr(o), _i(nint), C.c_char_p((path + " ").encode()))
        check()
        return o

    def autotune(self):
        """Time every lane-group size of every class on the last Fock build's
        quartet lists and keep the fastest (qb_autotune_classes)."""
        g = np.zeros(1024, dtype=np.int32)
        lib().qb_autotune_classes(_ptr(g), 1024)
        check()
        return g

    def autotune_grad(self):
        """Time the lanes-per-quartet sizes of the light gradient classes on
        the last gradient call's lists and keep the fastest (qb_autotune_grad)."""
        g = np.zeros(1024, dtype=np.int32)
        lib().qb_autotune_grad(_ptr(g), 1024)
        check()
        return g

    def set_grad_groups(self, groups, fp32=False):
        """Set every gradient class's lanes per quartet (qb_set_grad_groups)."""
        g = np.ascontiguousarray(groups, dtype=np.int32)
        lib().qb_set_grad_groups(_ptr(g), C.c_int(len(g)), C.c_int(1 if fp32 else 0))
        check()

    def set_class_groups(self, groups, fp32=False):
        """Set every class's launch variant (qb_set_class_groups)."""
        g = np.ascontiguousarray(groups, dtype=np.int32)
        lib().qb_set_class_groups(_ptr(g), C.c_int(len(g)), C.c_int(1 if fp32 else 0))
        check()

    @staticmethod
    def class_variants(cls, fp32=False):
        """The launch variants of class cls (qb_class_variants)."""
        codes = np.zeros(32, dtype=np.int32)
        n = lib().qb_class_variants(C.c_int(cls), C.c_int(1 if fp32 else 0), _ptr(codes), C.c_int(32))
        return [int(x) for x in codes[:n]]

    def oneint(self):
        """(S, H): the overlap of fullx and the core Hamiltonian of get1e."""
        n = self.nbasis
        S = np.zeros((n, n), order="F")
        H = np.zeros((n, n), order="F")
        r = lib()
        r.gpu_get_overlap_(_ptr(S))
        r.gpu_get1e_(_ptr(H))
        check()
        return S, H

    def grad1e(self, dense, wdense, grad_in=None):
        """grad_in + nuclear-repulsion and one-electron gradient (3 natom)."""
        na = len(self.basis.first_basis_function)
        g = np.zeros(3 * na) if grad_in is None else np.array(grad_in, dtype=np.float64).ravel(order="F").copy()
        d = np.asfortranarray(dense, dtype=np.float64)
        w = np.asfortranarray(wdense, dtype=np.float64)
        lib().gpu_grad1e_(_ptr(g), _ptr(d), _ptr(w))
        check()
        return g

    def getxc(self, O, dense, sigrad2, method=1, isg=1, Eelxc=0.0, aelec=0.0, belec=0.0):
        """QUICK's DFT step (src/dft.f90:893-899): upload_method / calculated +
        gpu_getxc_.  Returns (O + V_xc symmetrised, Eelxc, aelec, belec), the
        three scalars accumulated onto the given inputs."""
        r = lib()
        o = np.array(O, order="F", dtype=np.float64)
        co = np.zeros((1,), dtype=np.float64)
        d = np.asfortranarray(dense, dtype=np.float64)
        sg = np.ascontiguousarray(sigrad2, dtype=np.float64)
        e, a, b = C.c_double(Eelxc), C.c_double(aelec), C.c_double(belec)
        r.gpu_upload_method_(_i(method))
        r.gpu_upload_calculated_(_ptr(o), _ptr(co), _ptr(co), _ptr(d))
        r.gpu_getxc_(_i(isg), _ptr(sg), C.byref(e), C.byref(a), C.byref(b), _ptr(o))
        check()
        return o, e.value, a.value, b.value

    def xc_stats(self):
        n, c, a, b = C.c_longlong(0), C.c_longlong(0), C.c_double(0), C.c_double(0)
        lib().qb_last_xc_stats(C.byref(n), C.byref(c), C.byref(a), C.byref(b))
        x, y, z = C.c_double(0), C.c_double(0), C.c_double(0)
        lib().qb_last_xc_work(C.byref(x), C.byref(y), C.byref(z))
        return dict(npts=n.value, nchunks=c.value, ms=a.value, ms_grid=b.value, alg_bytes=x.value,
                    alg_flops=y.value, gemm_flops=z.value)

    def xc_grid(self):
        """(npts, 4) array of the kept grid points: x, y, z, weight."""
        r = lib()
        r.qb_xc_grid.restype = C.c_longlong
        n = r.qb_xc_grid(None, C.c_longlong(0))
        out = np.zeros((max(n, 1), 4))
        r.qb_xc_grid(_ptr(out), C.c_longlong(n))
        check()
        return out[:n]

    def set_mixed_precision(self, cut):
        """Quartets with Y_ab Y_cd DNMax below cut run in FP32 (0: all FP64)."""
        lib().qb_set_mixed_precision(C.c_double(cut))
        check()

    def fock_split(self):
        a, b = C.c_longlong(0), C.c_longlong(0)
        lib().qb_last_fock_split(C.byref(a), C.byref(b))
        return dict(fp64=a.value, fp32=b.value)

    def grad_stats(self):
        q, a = C.c_longlong(0), C.c_double(0)
        lib().qb_last_grad_stats(C.byref(q), C.byref(a))
        return dict(quartets=q.value, ms=a.value)

    def fock_stats(self):
        q, a, b = C.c_longlong(0), C.c_double(0), C.c_double(0)
        lib().qb_last_fock_stats(C.byref(q), C.byref(a), C.byref(b))
        return dict(quartets=q.value, ms_eri=a.value, ms_screen=b.value)

    def pairlist(self):
        cap = 1 << 24
        xy = np.zeros(2 * cap, dtype=np.int32)
        q = np.zeros(1 << 20, dtype=np.int32)
        qn = np.zeros(1 << 20, dtype=np.int32)
        f, ff = C.c_int(0), C.c_int(0)
        n = lib().qb_get_pairlist(_ptr(xy), cap, _ptr(q), _ptr(qn), 1 << 20, C.byref(f), C.byref(ff))
        check()
        nq = sum(int(self.basis.Qfinal[s] - self.basis.Qstart[s] + 1) for s in range(self.basis.nshell))
        return dict(pairs=xy[:2 * n].reshape(n, 2).copy(), fStart=f.value, ffStart=ff.value,
                    sorted_Q=q[:nq].copy(), sorted_Qnumber=qn[:nq].copy())

    def close(self):
        lib().gpu_shutdown_()


def xc_functional(method, rho, sigma):
    """The closed-shell functional on the GPU at arrays rho (total density)
    and sigma = |grad rho|^2: returns (f, df/drho, 4 df/dsigma)."""
    r = lib()
    rho = np.ascontiguousarray(rho, dtype=np.float64)
    sigma = np.ascontiguousarray(sigma, dtype=np.float64)
    out = np.zeros(3 * rho.size)
    r.qb_xc_functional(C.c_int(method), C.c_int(rho.size), _ptr(rho), _ptr(sigma), _ptr(out))
    check()
    out = out.reshape(-1, 3)
    return out[:, 0].copy(), out[:, 1].copy(), out[:, 2].copy()


def build_pairlist_host(basis, YCutoff):
    """QUICK's pair-list construction on the host (no GPU needed)."""
    sq, sqn = [], []
    for L in range(4):
        for s in range(basis.nshell):
            if basis.Qstart[s] <= L <= basis.Qfinal[s]:
                sq.append(s)
                sqn.append(L)
    sq = np.array(sq, dtype=np.int32)
    sqn = np.array(sqn, dtype=np.int32)
    kp = np.ascontiguousarray(basis.kprim, dtype=np.int32)
    Y = np.asfortranarray(YCutoff, dtype=np.float64)
    cap = len(sq) * len(sq)
    xy = np.zeros(2 * cap, dtype=np.int32)
    f, ff = C.c_int(0), C.c_int(0)
    n = lib().qb_build_pairlist_host(len(sq), _ptr(sq), _ptr(sqn), _ptr(kp), basis.nshell, _ptr(Y), _ptr(xy), cap,
                                     C.byref(f), C.byref(ff))
    return dict(pairs=xy[:2 * n].reshape(n, 2).copy(), fStart=f.value, ffStart=ff.value,
                sorted_Q=sq, sorted_Qnumber=sqn)
