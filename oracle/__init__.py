"""CPU oracle for QUICK's direct-SCF two-electron path.

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and
bench.py's cpu_baseline / reference legs, never by the quick_b200 package.

Two checkers live here:
  * ``liboracle.so`` (oracle.c): this project's plain-C restatement of the
    reference's algorithm;
  * ``libquickref.so`` (build_ref.py): QUICK's own CUDA bridge and kernels
    (src/cuda/gpu.cu, gpu_get2e.cu, gpu_getxc.cu) compiled as host code and
    driven through QUICK's own ``gpu_*_`` entry points, in the call order of
    src/main.f90:81-177 and src/hfoperator.f90:76-104;
  * ``gpu/libquickref.so`` (build_ref.py --gpu): the same QUICK sources built
    unchanged by nvcc for sm_100a and driven the same way on a GPU -- QUICK's
    own GPU path, the GPU-side baseline and a second checker.
"""
import contextlib
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIBDIR = os.path.join(HERE, "_ref")

_P = C.c_void_p


def _ptr(a):
    return a.ctypes.data_as(_P)


class _OBasis(C.Structure):
    _fields_ = [("natom", C.c_int), ("nbasis", C.c_int), ("nshell", C.c_int), ("jbasis", C.c_int),
                ("xyz", _P), ("kstart", _P), ("katom", _P), ("kprim", _P), ("Ksumtype", _P),
                ("Qstart", _P), ("Qfinal", _P), ("Qsbasis", _P), ("Qfbasis", _P), ("KLMN", _P),
                ("gccoeff", _P), ("gcexpo", _P), ("cons", _P)]


def build_oracle():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(LIBDIR, "liboracle.so")
        if not os.path.exists(path):
            build_oracle()
        _lib = C.CDLL(path)
        _lib.oracle_fock.restype = C.c_long
        _lib.oracle_shell_quartet.restype = C.c_long
    return _lib


class OracleInputs:
    """Keeps the numpy arrays alive behind the C struct."""

    def __init__(self, basis, xyz_bohr):
        b = basis
        self.keep = dict(
            xyz=np.asfortranarray(xyz_bohr, dtype=np.float64),
            kstart=np.ascontiguousarray(b.kstart, dtype=np.int32),
            katom=np.ascontiguousarray(b.katom, dtype=np.int32),
            kprim=np.ascontiguousarray(b.kprim, dtype=np.int32),
            Ksumtype=np.ascontiguousarray(b.Ksumtype, dtype=np.int32),
            Qstart=np.ascontiguousarray(b.Qstart, dtype=np.int32),
            Qfinal=np.ascontiguousarray(b.Qfinal, dtype=np.int32),
            Qsbasis=np.asfortranarray(b.Qsbasis, dtype=np.int32),
            Qfbasis=np.asfortranarray(b.Qfbasis, dtype=np.int32),
            KLMN=np.asfortranarray(b.KLMN, dtype=np.int32),
            gccoeff=np.asfortranarray(b.gccoeff),
            gcexpo=np.asfortranarray(b.gcexpo),
            cons=np.ascontiguousarray(b.cons))
        k = self.keep
        self.s = _OBasis(b.natom, b.nbasis, b.nshell, b.jbasis, *[_ptr(k[n]) for n in (
            "xyz", "kstart", "katom", "kprim", "Ksumtype", "Qstart", "Qfinal", "Qsbasis",
            "Qfbasis", "KLMN", "gccoeff", "gcexpo", "cons")])
        self.basis = basis


def boys(mmax, T):
    F = np.zeros(mmax + 1)
    lib().oracle_boys(C.c_int(mmax), C.c_double(T), _ptr(F))
    return F


def schwarz(basis, xyz_bohr):
    """YCutoff (nshell x nshell) and cutPrim (jbasis x jbasis), Fortran order."""
    inp = OracleInputs(basis, xyz_bohr)
    Y = np.zeros((basis.nshell, basis.nshell), order="F")
    cp = np.zeros((basis.jbasis, basis.jbasis), order="F")
    lib().oracle_schwarz(C.byref(inp.s), _ptr(Y), _ptr(cp))
    return Y, cp


def cutmatrix(basis, dense):
    cm = np.zeros((basis.nshell, basis.nshell), order="F")
    inp = OracleInputs(basis, np.zeros((3, basis.natom), order="F"))
    d = np.asfortranarray(dense)
    lib().oracle_cutmatrix(C.byref(inp.s), _ptr(d), _ptr(cm))
    return cm


def fock(basis, xyz_bohr, YCutoff, cutPrim, cutMatrix, dense, integral_cutoff, prim_limit,
         hybrid=1.0, O=None):
    """O + G(D) as QUICK's get2e returns it; also the quartet counts."""
    inp = OracleInputs(basis, xyz_bohr)
    n = basis.nbasis
    O = np.zeros((n, n), order="F") if O is None else np.array(O, order="F", dtype=np.float64)
    Y, cp, cm, d = (np.asfortranarray(a, dtype=np.float64) for a in (YCutoff, cutPrim, cutMatrix, dense))
    npq, nint = C.c_long(0), C.c_long(0)
    nq = lib().oracle_fock(C.byref(inp.s), _ptr(Y), _ptr(cp), _ptr(cm), _ptr(d),
                           C.c_double(integral_cutoff), C.c_double(prim_limit), C.c_double(hybrid),
                           _ptr(O), C.byref(npq), C.byref(nint))
    return O, dict(quartets=int(nq), prim_quartets=int(npq.value), integrals=int(nint.value))


def grad2e(basis, xyz_bohr, YCutoff, cutPrim, cutMatrix, dense, integral_cutoff, prim_limit, hybrid=1.0):
    """Two-electron part of the nuclear gradient, (3, natom) flattened like QUICK's."""
    inp = OracleInputs(basis, xyz_bohr)
    g = np.zeros(3 * basis.natom)
    Y, cp, cm, d = (np.asfortranarray(a, dtype=np.float64) for a in (YCutoff, cutPrim, cutMatrix, dense))
    lib().oracle_grad(C.byref(inp.s), _ptr(Y), _ptr(cp), _ptr(cm), _ptr(d), C.c_double(integral_cutoff),
                      C.c_double(prim_limit), C.c_double(hybrid), _ptr(g))
    return g


def energy2e(basis, xyz_bohr, YCutoff, cutPrim, cutMatrix, dense, integral_cutoff, prim_limit, hybrid=1.0):
    """E2 = Tr[D G(D)] / 2 from the oracle's Fock build."""
    G, _ = fock(basis, xyz_bohr, YCutoff, cutPrim, cutMatrix, dense, integral_cutoff, prim_limit, hybrid)
    return 0.5 * float(np.sum(np.asarray(dense) * G))


def ref_grad(grad_in, dense, cutMatrix, integral_cutoff, prim_limit, grad_cutoff=1e-7):
    """QUICK's gradient path (src/gradient.f90:279-286): upload_calculated,
    upload_cutoff, upload_grad, gpu_grad_.  Returns grad_in + the 2e gradient."""
    r = ref_lib()
    n = dense.shape[0]
    o = np.zeros((n, n), order="F")
    co = np.zeros((n, n), order="F")
    d = np.array(dense, order="F", dtype=np.float64)
    cm = np.array(cutMatrix, order="F", dtype=np.float64)
    g = np.array(grad_in, dtype=np.float64)
    with _quiet():
        r.gpu_upload_calculated_(_ptr(o), _ptr(co), _ptr(co), _ptr(d))
        r.gpu_upload_cutoff_(_ptr(cm), _d(integral_cutoff), _d(prim_limit), None)
        r.gpu_upload_grad_(_ptr(g), _d(grad_cutoff))
        r.gpu_grad_(_ptr(g))
    return g


def shell_quartet(basis, xyz_bohr, ii, jj, kk, ll, I, J, K, L):
    """Contracted (ab|cd) block (0-based shells) without screening."""
    inp = OracleInputs(basis, xyz_bohr)
    out = np.zeros(10 ** 4)
    lib().oracle_shell_quartet(C.byref(inp.s), ii, jj, kk, ll, I, J, K, L, C.c_double(-1.0), None,
                               C.c_double(0.0), -1, _ptr(out))
    return out


# ------------------------------------------------------------ QUICK itself
_ref = None


_ref_spdf = None


_ref_variants = {}


class _O1Basis(C.Structure):
    _fields_ = [("natom", C.c_int), ("nbasis", C.c_int), ("nshell", C.c_int), ("maxcontract", C.c_int),
                ("xyz", _P), ("chg", _P), ("ncontract", _P), ("itype", _P), ("ncenter", _P),
                ("aexp", _P), ("dcoeff", _P), ("katom", _P), ("kprim", _P), ("Ksumtype", _P),
                ("Qstart", _P), ("Qfinal", _P), ("Qsbasis", _P), ("Qfbasis", _P), ("KLMN", _P),
                ("gccoeff", _P), ("gcexpo", _P), ("cons", _P)]


class OneElectronInputs:
    """The arrays oracle_1e.c reads (QUICK's per-function and per-shell basis
    arrays, coordinates and nuclear charges), kept alive behind the struct."""

    def __init__(self, basis, mol):
        b = basis
        I32 = np.int32
        self.keep = dict(
            xyz=np.asfortranarray(mol.xyz_bohr, dtype=np.float64),
            chg=np.ascontiguousarray(mol.atomic_numbers, dtype=np.float64),
            ncontract=np.ascontiguousarray(b.ncontract, dtype=I32),
            itype=np.asfortranarray(b.itype, dtype=I32),
            ncenter=np.ascontiguousarray(b.ncenter, dtype=I32),
            aexp=np.asfortranarray(b.aexp, dtype=np.float64),
            dcoeff=np.asfortranarray(b.dcoeff, dtype=np.float64),
            katom=np.ascontiguousarray(b.katom, dtype=I32),
            kprim=np.ascontiguousarray(b.kprim, dtype=I32),
            Ksumtype=np.ascontiguousarray(b.Ksumtype, dtype=I32),
            Qstart=np.ascontiguousarray(b.Qstart, dtype=I32),
            Qfinal=np.ascontiguousarray(b.Qfinal, dtype=I32),
            Qsbasis=np.asfortranarray(b.Qsbasis, dtype=I32),
            Qfbasis=np.asfortranarray(b.Qfbasis, dtype=I32),
            KLMN=np.asfortranarray(b.KLMN, dtype=I32),
            gccoeff=np.asfortranarray(b.gccoeff),
            gcexpo=np.asfortranarray(b.gcexpo),
            cons=np.ascontiguousarray(b.cons))
        k = self.keep
        self.s = _O1Basis(mol.natom, b.nbasis, b.nshell, b.maxcontract, *[_ptr(k[n]) for n in (
            "xyz", "chg", "ncontract", "itype", "ncenter", "aexp", "dcoeff", "katom", "kprim", "Ksumtype",
            "Qstart", "Qfinal", "Qsbasis", "Qfbasis", "KLMN", "gccoeff", "gcexpo", "cons")])


def oneint(basis, mol):
    """Overlap S and core Hamiltonian H = T + V (nbasis x nbasis, symmetric)."""
    inp = OneElectronInputs(basis, mol)
    n = basis.nbasis
    S = np.zeros((n, n), order="F")
    H = np.zeros((n, n), order="F")
    lib().oracle_oneint(C.byref(inp.s), _ptr(S), _ptr(H))
    return S, H


def enuc(mol):
    xyz = np.asfortranarray(mol.xyz_bohr, dtype=np.float64)
    chg = np.ascontiguousarray(mol.atomic_numbers, dtype=np.float64)
    f = lib().oracle_enuc
    f.restype = C.c_double
    return float(f(C.c_int(mol.natom), _ptr(xyz), _ptr(chg)))


def grad1e(basis, mol, dense, wdense):
    """Nuclear-repulsion and one-electron parts of the RHF gradient, (3 natom)."""
    inp = OneElectronInputs(basis, mol)
    g = np.zeros(3 * mol.natom)
    d = np.asfortranarray(dense, dtype=np.float64)
    w = np.asfortranarray(wdense, dtype=np.float64)
    lib().oracle_grad1e(C.byref(inp.s), _ptr(d), _ptr(w), _ptr(g))
    return g


def _ref_dir(spdf):
    """spdf: False (default build), True (CUDA_SPDF: QUICK's f-shell kernels)
    or "boys" (CUDA_SPDF with QUICK's FmT replaced by an accurate Boys
    function, build_ref.py --accurate-boys), or "gpu" (QUICK's sources built
    unchanged by nvcc for sm_100a, build_ref.py --gpu: QUICK's own GPU path,
    which needs a GPU; it has no quartet counter and no host threads)."""
    return {False: LIBDIR, True: os.path.join(LIBDIR, "spdf"), "boys": os.path.join(LIBDIR, "spdf_boys"),
            "gpu": os.path.join(LIBDIR, "gpu")}[spdf]


def ref_available(spdf=False):
    return os.path.exists(os.path.join(_ref_dir(spdf), "libquickref.so"))


def ref_lib(spdf=False):
    """QUICK's host build (see _ref_dir for the variants)."""
    global _ref
    if spdf is False:
        if _ref is None:
            _ref = C.CDLL(os.path.join(LIBDIR, "libquickref.so"))
        return _ref
    if spdf not in _ref_variants:
        _ref_variants[spdf] = C.CDLL(os.path.join(_ref_dir(spdf), "libquickref.so"))
    return _ref_variants[spdf]


@contextlib.contextmanager
def _quiet():
    """QUICK's bridge prints every pair it sorts; silence fd 1 meanwhile."""
    import sys
    sys.stdout.flush()
    saved = os.dup(1)
    devnull = os.open(os.devnull, os.O_WRONLY)
    os.dup2(devnull, 1)
    try:
        yield
    finally:
        C.CDLL(None).fflush(None)
        os.dup2(saved, 1)
        os.close(saved)
        os.close(devnull)


@contextlib.contextmanager
def _capture(lines):
    """Like _quiet, but the text QUICK's bridge prints is kept: appended to
    the list ``lines`` when the block ends."""
    import sys
    import tempfile
    sys.stdout.flush()
    saved = os.dup(1)
    with tempfile.TemporaryFile(mode="w+b") as tmp:
        os.dup2(tmp.fileno(), 1)
        try:
            yield
        finally:
            C.CDLL(None).fflush(None)
            os.dup2(saved, 1)
            os.close(saved)
            tmp.seek(0)
            lines.extend(tmp.read().decode("latin-1").splitlines())


def ref_get2e_gpu_timed(O, dense, cutMatrix, integral_cutoff, prim_limit, method=0):
    """One Fock build through QUICK's GPU build (ref_lib("gpu")), the
    sequence of ref_get2e.  Returns (O, wall seconds of the four bridge
    calls, QUICK's own event time of its get2e_kernel launch in ms).  QUICK's
    stock configuration defines DEBUG, under which QUICK_SAFE_CALL brackets
    the launch with CUDA events and prints "this cycle:<ms> ms"
    (src/cuda/gpu_common.h:90-146); that line is read back here."""
    import time
    r = ref_lib("gpu")
    n = O.shape[0]
    o = np.array(O, order="F", dtype=np.float64)
    co = np.zeros((n, n), order="F")
    vec = np.zeros((n, n), order="F")
    d = np.array(dense, order="F", dtype=np.float64)
    cm = np.array(cutMatrix, order="F", dtype=np.float64)
    lines = []
    with _capture(lines):
        t0 = time.perf_counter()
        r.gpu_upload_method_(_i(method))
        r.gpu_upload_calculated_(_ptr(o), _ptr(co), _ptr(vec), _ptr(d))
        r.gpu_upload_cutoff_(_ptr(cm), _d(integral_cutoff), _d(prim_limit), None)
        r.gpu_get2e_(_ptr(o))
        wall = time.perf_counter() - t0
    kern = [float(x.split("this cycle:")[1].split("ms")[0]) for x in lines if "this cycle:" in x]
    if len(kern) != 1:
        raise RuntimeError("expected one timed QUICK launch, got %r" % (kern,))
    return o, wall, kern[0]


def ref_grad_gpu_timed(ngrad, dense, cutMatrix, integral_cutoff, prim_limit, grad_cutoff=1e-7):
    """QUICK's two-electron gradient through its GPU build, the sequence of
    ref_grad.  Returns (gradient, wall seconds of the four bridge calls, the
    sum of QUICK's own event times of its gradient launches in ms:
    getGrad_kernel and, with d shells, getGrad_kernel_spdf and _spdf2,
    src/cuda/gpu_get2e.cu:336-350)."""
    import time
    r = ref_lib("gpu")
    n = dense.shape[0]
    o = np.zeros((n, n), order="F")
    co = np.zeros((n, n), order="F")
    d = np.array(dense, order="F", dtype=np.float64)
    cm = np.array(cutMatrix, order="F", dtype=np.float64)
    g = np.zeros(ngrad)
    lines = []
    with _capture(lines):
        t0 = time.perf_counter()
        r.gpu_upload_calculated_(_ptr(o), _ptr(co), _ptr(co), _ptr(d))
        r.gpu_upload_cutoff_(_ptr(cm), _d(integral_cutoff), _d(prim_limit), None)
        r.gpu_upload_grad_(_ptr(g), _d(grad_cutoff))
        r.gpu_grad_(_ptr(g))
        wall = time.perf_counter() - t0
    kern = [float(x.split("this cycle:")[1].split("ms")[0]) for x in lines if "this cycle:" in x]
    return g, wall, float(sum(kern))


def ref_getxc_gpu_timed(dense, sigrad2, method=1, isg=1):
    """One XC quadrature through QUICK's GPU build, the sequence of
    ref_getxc.  Returns (O', Eelxc, aelec, wall seconds of the three bridge
    calls; gpu_getxc_ returns after its download)."""
    import time
    r = ref_lib("gpu")
    n = dense.shape[0]
    o = np.zeros((n, n), order="F")
    co = np.zeros((n, n), order="F")
    vec = np.zeros((n, n), order="F")
    d = np.array(dense, order="F", dtype=np.float64)
    sg = np.ascontiguousarray(sigrad2, dtype=np.float64)
    e, a, b = C.c_double(0.0), C.c_double(0.0), C.c_double(0.0)
    cm = np.zeros((max(_ref_nshell, 1),) * 2, order="F")
    with _quiet():
        r.gpu_upload_cutoff_(_ptr(cm), _d(1e-10), _d(1e-20), None)
        t0 = time.perf_counter()
        r.gpu_upload_method_(_i(method))
        r.gpu_upload_calculated_(_ptr(o), _ptr(co), _ptr(vec), _ptr(d))
        r.gpu_getxc_(_i(isg), _ptr(sg), C.byref(e), C.byref(a), C.byref(b), _ptr(o))
        wall = time.perf_counter() - t0
    return o, e.value, a.value, wall


def _i(v):
    return C.byref(C.c_int(int(v)))


def _d(v):
    return C.byref(C.c_double(float(v)))


_ref_nshell = 0


def ref_upload_molecule(mol, basis, YCutoff, cutPrim, threads=None, spdf=False, device=0):
    """QUICK's start-up upload sequence (src/main.f90:84-177); device: the
    CUDA device of the "gpu" build (gpu_set_device_, src/cuda/gpu.cu:18)."""
    global _ref_nshell
    _ref_nshell = basis.nshell
    r = ref_lib(spdf)
    if threads and spdf != "gpu":
        r.qref_set_threads(int(threads))
    b = basis
    keep = []

    def arr(a, dt):
        x = np.asfortranarray(a, dtype=dt)
        keep.append(x)
        return _ptr(x)

    with _quiet():
        r.qref_reset()
        if spdf == "gpu":
            r.gpu_set_device_(_i(device))
        r.gpu_init_()
        r.gpu_setup_(_i(mol.natom), _i(b.nbasis), _i(mol.n_electrons), _i(mol.mult), _i(mol.charge),
                     _i(len(set(mol.symbols))))
        r.gpu_upload_xyz_(arr(mol.xyz_bohr, np.float64))
        r.gpu_upload_atom_and_chg_(arr(mol.atomic_numbers, np.int32),
                                   arr(mol.atomic_numbers.astype(np.float64), np.float64))
        I32, F64 = np.int32, np.float64
        r.gpu_upload_basis_(_i(b.nshell), _i(b.nprim), _i(b.jshell), _i(b.jbasis), _i(b.maxcontract),
                            arr(b.ncontract, I32), arr(b.itype, I32), arr(b.aexp, F64), arr(b.dcoeff, F64),
                            arr(b.first_basis_function, I32), arr(b.last_basis_function, I32),
                            arr(b.first_shell_basis_function, I32), arr(b.last_shell_basis_function, I32),
                            arr(b.ncenter, I32), arr(b.kstart, I32), arr(b.katom, I32), arr(b.ktype, I32),
                            arr(b.kprim, I32), arr(b.kshell, I32), arr(b.Ksumtype, I32), arr(b.Qnumber, I32),
                            arr(b.Qstart, I32), arr(b.Qfinal, I32), arr(b.Qsbasis, I32), arr(b.Qfbasis, I32),
                            arr(b.gccoeff, F64), arr(b.cons, F64), arr(b.gcexpo, F64), arr(b.KLMN, I32))
        r.gpu_upload_cutoff_matrix_(arr(YCutoff, F64), arr(cutPrim, F64))
    return keep


def ref_pairlist():
    r = ref_lib()
    cap = 1 << 24
    xy = np.zeros(2 * cap, dtype=np.int32)
    f, ff = C.c_int(0), C.c_int(0)
    n = r.qref_pairlist(_ptr(xy), cap, C.byref(f), C.byref(ff))
    q = np.zeros(1 << 20, dtype=np.int32)
    qn = np.zeros(1 << 20, dtype=np.int32)
    nq = r.qref_sorted_q(_ptr(q), _ptr(qn), 1 << 20)
    return dict(pairs=xy[:2 * n].reshape(n, 2).copy(), fStart=f.value, ffStart=ff.value,
                sorted_Q=q[:nq].copy(), sorted_Qnumber=qn[:nq].copy())


def ref_quartet_counts(spdf=False):
    """Shell quartets of the last QUICK Fock builds since ref_get2e reset the
    counter: (raw, unique).  raw counts QUICK's iclass calls
    (gpu_get2e_subs.h:327-336: ordered pair-pairs with ii <= kk that pass both
    Schwarz tests); unique counts the same walk once per unordered pair of
    shell pairs, without the (p,s) copy of an sp shell's self-pair -- the
    metric's unit."""
    r = ref_lib(spdf)
    raw, uniq = C.c_longlong(0), C.c_longlong(0)
    r.qref_quartet_counts(C.byref(raw), C.byref(uniq))
    return raw.value, uniq.value


def ref_get2e(O, dense, cutMatrix, integral_cutoff, prim_limit, method=0, spdf=False):
    """One QUICK Fock build: upload_method/calculated/cutoff + gpu_get2e_
    (src/hfoperator.f90:76-98).  Returns the new O; ref_quartet_counts()
    then gives its shell-quartet counts."""
    r = ref_lib(spdf)
    if spdf != "gpu":
        r.qref_reset_counts()
    n = O.shape[0]
    o = np.array(O, order="F", dtype=np.float64)
    co = np.zeros((n, n), order="F")
    vec = np.zeros((n, n), order="F")
    d = np.array(dense, order="F", dtype=np.float64)
    cm = np.array(cutMatrix, order="F", dtype=np.float64)
    with _quiet():
        r.gpu_upload_method_(_i(method))
        r.gpu_upload_calculated_(_ptr(o), _ptr(co), _ptr(vec), _ptr(d))
        r.gpu_upload_cutoff_(_ptr(cm), _d(integral_cutoff), _d(prim_limit), None)
        r.gpu_get2e_(_ptr(o))
    return o


def ref_getxc(O, dense, sigrad2, method=1, isg=1, Eelxc=0.0, aelec=0.0, belec=0.0, threads=None):
    """One QUICK XC quadrature: upload_method / upload_calculated + gpu_getxc_
    (src/dft.f90:893-899), run by QUICK's own getxc_kernel compiled for the
    host.  Needs ref_upload_molecule first.  Returns (O', Eelxc, aelec, belec)."""
    r = ref_lib()
    r.qref_set_threads(int(threads or os.cpu_count() or 1))
    n = O.shape[0]
    o = np.array(O, order="F", dtype=np.float64)
    co = np.zeros((n, n), order="F")
    vec = np.zeros((n, n), order="F")
    d = np.array(dense, order="F", dtype=np.float64)
    sg = np.ascontiguousarray(sigrad2, dtype=np.float64)
    e, a, b = C.c_double(Eelxc), C.c_double(aelec), C.c_double(belec)
    # gpu_upload_cutoff_ is where QUICK's bridge sets its DMCutoff (1e-9,
    # src/cuda/gpu.cu:370); the cut matrix itself is not read by the XC path.
    cm = np.zeros((max(_ref_nshell, 1),) * 2, order="F")
    with _quiet():
        r.gpu_upload_method_(_i(method))
        r.gpu_upload_calculated_(_ptr(o), _ptr(co), _ptr(vec), _ptr(d))
        r.gpu_upload_cutoff_(_ptr(cm), _d(1e-10), _d(1e-20), None)
        r.qref_set_virtual_threads(1024)
        try:
            r.gpu_getxc_(_i(isg), _ptr(sg), C.byref(e), C.byref(a), C.byref(b), _ptr(o))
        finally:
            r.qref_set_virtual_threads(0)
    return o, e.value, a.value, b.value


def ref_functional(method, rho, sigma):
    """QUICK's functional routines at closed-shell points (total density rho,
    sigma = |grad rho|^2): returns (f, dfdr, dot) arrays."""
    r = ref_lib()
    f, fr, fs = C.c_double(), C.c_double(), C.c_double()
    rho = np.asarray(rho, dtype=np.float64).ravel()
    sigma = np.asarray(sigma, dtype=np.float64).ravel()
    out = np.zeros((rho.size, 3))
    for k in range(rho.size):
        r.qref_functional(C.c_int(method), C.c_double(rho[k]), C.c_double(sigma[k]), C.byref(f), C.byref(fr),
                          C.byref(fs))
        out[k] = f.value, fr.value, fs.value
    return out[:, 0], out[:, 1], out[:, 2]
