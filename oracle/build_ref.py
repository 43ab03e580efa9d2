"""Build ``oracle/_ref/libquickref.so``: QUICK's own CUDA bridge and kernels
compiled as host code, used only as the checker for this package.

The sources are read where they lie in the QUICK tree (``src/cuda``); the
shim in ``oracle/ref_shim`` supplies a host stand-in for the CUDA runtime and
the launch geometry.  Build outputs go to ``oracle/_ref`` only.

    python oracle/build_ref.py [--quick-root DIR] [--spdf] [--accurate-boys]
    python oracle/build_ref.py [--quick-root DIR] --gpu

--gpu compiles the same QUICK sources unchanged with nvcc for sm_100a into
``oracle/_ref/gpu/libquickref.so`` (QUICK's spd build, its own flags -O3
-use_fast_math from makein/make.in.gnu.cuda:52, plus a register cap so that
its 512-thread blocks can launch): QUICK's GPU path, timed on the B200
beside this package as a baseline.

The QUICK tree is DIR, else the environment variable QUICK_ROOT, else
/root/reference (quick_root()).
"""
import argparse
import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
SHIM = os.path.join(HERE, "ref_shim")
OUT = os.path.join(HERE, "_ref")
CUDA_INC = "/usr/local/cuda/include"
DEFAULT_QUICK_ROOT = "/root/reference"


def quick_root():
    """The QUICK source tree: $QUICK_ROOT, else the default location."""
    return os.environ.get("QUICK_ROOT") or DEFAULT_QUICK_ROOT


def build(quick_root, spdf=False, accurate_boys=False, jobs=8, opt="-O2"):
    """spdf: QUICK's f-shell kernels too (CUDA_SPDF), into oracle/_ref/spdf/.
    accurate_boys (with spdf): QUICK's kernels with its Boys function FmT
    replaced by an accurate one (qref_boys_accurate in ref_kernels.cpp), into
    oracle/_ref/spdf_boys/ -- QUICK's upward recursion loses most digits for
    small T and high m, and this build separates that from everything else."""
    if accurate_boys:
        OUT = os.path.join(HERE, "_ref", "spdf_boys")
    else:
        OUT = os.path.join(HERE, "_ref", "spdf") if spdf else os.path.join(HERE, "_ref")
    src = os.path.join(quick_root, "src", "cuda")
    if not os.path.isdir(src):
        raise FileNotFoundError("QUICK sources not found at %s" % src)
    os.makedirs(os.path.join(OUT, "inc"), exist_ok=True)
    # QUICK's headers include "../config.h" relative to src/cuda; with
    # -I_ref/inc that resolves to _ref/config.h.
    with open(os.path.join(SHIM, "config.h")) as fh:
        cfg = fh.read()
    if spdf:
        cfg += "#define CUDA_SPDF\n"
    with open(os.path.join(OUT, "config.h"), "w") as fh:
        fh.write(cfg)
    # gpu_getxc.cu: replace its one bare kernel launch (see ref_xc.cpp)
    with open(os.path.join(src, "gpu_getxc.cu")) as fh:
        xc = fh.read()
    xc, n = re.subn(r"getxc_kernel<<<[^;]*?>>>\(\);", 'qref_launch("getxc_kernel<<<>>>");', xc)
    assert n == 1, "expected one getxc_kernel launch"
    with open(os.path.join(OUT, "gpu_getxc_host.cu"), "w") as fh:
        fh.write(xc)
    # build-directory copies: gpu_get2e.cu (so that its quoted includes look
    # here first) and gpu_get2e_subs.h with a call of qref_count_quartet
    # beside the spd walk's iclass call (the shell-quartet counter of the
    # metric); with accurate_boys, QUICK's FmT renamed and an FmT that calls
    # the accurate Boys function in its place
    with open(os.path.join(src, "gpu_get2e.cu")) as fh:
        g2 = fh.read()
    with open(os.path.join(OUT, "gpu_get2e.cu"), "w") as fh:
        fh.write(g2)
    with open(os.path.join(src, "gpu_get2e_subs.h")) as fh:
        sub = fh.read()
    call = "iclass(iii, jjj, kkk, lll, ii, jj, kk, ll, DNMax);"
    assert sub.count(call) == 1, "expected one spd iclass call"
    sub = sub.replace(call, "qref_count_quartet(a, b, II, JJ, KK, LL, ii, kk); " + call)
    if accurate_boys:
        decl = "__device__ __forceinline__ void FmT(int MaxM, QUICKDouble X, QUICKDouble* YVerticalTemp)"
        assert sub.count(decl) == 1, "expected one FmT definition"
        sub = sub.replace(decl, "__device__ __forceinline__ void FmT(int MaxM, QUICKDouble X, QUICKDouble* YVerticalTemp)\n"
                                "{ qref_boys_accurate(MaxM, X, YVerticalTemp); }\n"
                                "__device__ __forceinline__ void FmT_quick(int MaxM, QUICKDouble X, QUICKDouble* YVerticalTemp)")
    with open(os.path.join(OUT, "gpu_get2e_subs.h"), "w") as fh:
        fh.write(sub)
    flags = [opt, "-fPIC", "-std=c++17", "-w", "-include", os.path.join(SHIM, "qref_shim.h"),
             "-I" + SHIM, "-I" + os.path.join(OUT, "inc"), "-I" + OUT, "-I" + src, "-I" + CUDA_INC]
    units = ["ref_bridge", "ref_kernels", "ref_type", "ref_xc"]
    objs = []

    def cc(u):
        o = os.path.join(OUT, u + ".o")
        cmd = ["g++"] + flags + ["-c", os.path.join(SHIM, u + ".cpp"), "-o", o]
        subprocess.run(cmd, check=True)
        return o

    with ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(cc, units))
    fo = os.path.join(OUT, "fake_cudart.o")
    subprocess.run(["g++", opt, "-fPIC", "-std=c++17", "-I" + CUDA_INC, "-c",
                    os.path.join(SHIM, "fake_cudart.cpp"), "-o", fo], check=True)
    lib = os.path.join(OUT, "libquickref.so")
    subprocess.run(["g++", "-shared", "-Wl,-Bsymbolic", "-o", lib] + objs + [fo, "-lpthread"], check=True)
    return lib


def build_gpu(quick_root, jobs=4):
    """QUICK's bridge and kernels (src/cuda/gpu.cu, gpu_type.cu, gpu_get2e.cu,
    gpu_getxc.cu; the units of src/cuda/Makefile:16-19) built by nvcc for
    sm_100a, unchanged, into oracle/_ref/gpu/libquickref.so."""
    out = os.path.join(HERE, "_ref", "gpu")
    src = os.path.join(quick_root, "src", "cuda")
    if not os.path.isdir(src):
        raise FileNotFoundError("QUICK sources not found at %s" % src)
    os.makedirs(os.path.join(out, "inc"), exist_ok=True)
    # QUICK's own CUDA configuration, as its Makefile copies it to src/config.h
    # (Makefile:181 copies config/config.cuda.h; it defines DEBUG, which QUICK_SAFE_CALL's
    # event timer around every kernel launch needs, gpu_common.h:90-134)
    with open(os.path.join(quick_root, "src", "config", "config.cuda.h")) as fh:
        cfg = fh.read()
    with open(os.path.join(out, "config.h"), "w") as fh:
        fh.write(cfg)
    nvcc = os.path.join(os.environ.get("CUDA_HOME", "/usr/local/cuda"), "bin", "nvcc")
    # -maxrregcount=128: QUICK launches its kernels with 512 threads per block
    # (gpu_common.h:180-190, gpu_init_) and declares no launch bounds; left
    # alone, ptxas gives get2e_kernel 255 registers on sm_100a and such a
    # block cannot launch (65,536 registers per SM).  QUICK's own flag line
    # for its first GPUs capped registers the same way (-maxrregcount=63,
    # makein/make.in.gnu.cuda:50).
    flags = ["-O3", "-use_fast_math", "-m64", "-maxrregcount=128", "-gencode", "arch=compute_100a,code=sm_100a",
             "-w", "-Xptxas", "-v",
             "-Xcompiler", "-fPIC", "-I" + os.path.join(out, "inc"), "-I" + out, "-I" + src]
    units = [os.path.join(SHIM, "gpu_bridge.cu")] + [os.path.join(src, u) for u in
                                                    ("gpu_type.cu", "gpu_get2e.cu", "gpu_getxc.cu")]

    def cc(u):
        o = os.path.join(out, os.path.basename(u).replace(".cu", ".o"))
        with open(o.replace(".o", ".ptxas.txt"), "w") as log:   # resource usage per kernel
            subprocess.run([nvcc] + flags + ["-c", u, "-o", o], check=True, stderr=log)
        return o

    with ThreadPoolExecutor(jobs) as ex:
        objs = list(ex.map(cc, units))
    lib = os.path.join(out, "libquickref.so")
    subprocess.run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-Xlinker", "-Bsymbolic",
                    "-o", lib] + objs, check=True)
    return lib


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--quick-root", default=None)
    ap.add_argument("--spdf", action="store_true")
    ap.add_argument("--accurate-boys", action="store_true")
    ap.add_argument("--gpu", action="store_true")
    a = ap.parse_args()
    if a.gpu:
        print(build_gpu(a.quick_root or quick_root()))
        sys.exit(0)
    print(build(a.quick_root or quick_root(), a.spdf or a.accurate_boys, a.accurate_boys))
