"""Build ``quick_b200/_lib/libquickb200.so`` (sm_100a) in-tree.

Generates the per-class kernels (csrc/gen_eri.py), compiles every CUDA
source with nvcc for sm_100a in parallel and links one shared library with
the CUDA runtime linked statically.  Rebuilds only what changed.

    python -m quick_b200.build [--lmax 2] [--jobs 8]
"""
import argparse
import os
import re
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
GEN = os.path.join(CSRC, "gen")
OBJ = os.path.join(HERE, "_build")
LIBDIR = os.path.join(HERE, "_lib")
LIB = os.path.join(LIBDIR, "libquickb200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr",
         "-I" + CSRC, "-I" + os.path.join(HERE, "..", "include")]


def _extra_flags(src):
    """Per-file ptxas options.  For the generated Fock classes with total
    angular momentum >= 6, and the gradient classes with total angular
    momentum >= 4, ptxas at its default -O3 falls back to a 32-register
    allocation that spills nearly everything (grad_2110: 32 registers and a
    10.5 KB stack frame); -O1 keeps 255 registers and spills about a third as
    much (measured with -Xptxas -v for every class)."""
    b = os.path.basename(src)
    for pre, lim in (("eri_", 6), ("eri32_", 6), ("grad_", 4), ("grad32_", 4)):
        if b.startswith(pre) and b[len(pre):len(pre) + 4].isdigit():
            if sum(int(ch) for ch in b[len(pre):len(pre) + 4]) >= lim:
                return ["-Xptxas", "-O1"]
    return []


# f classes with straight-line kernels: total angular momentum up to this
# (gen_eri.py, F_MAX_L)
F_MAX_L = 8


def _generated_class(src):
    """A generated straight-line class file (Fock, FP32 Fock, gradient)."""
    b = os.path.basename(src)
    return any(b.startswith(pre) and b[len(pre):len(pre) + 4].isdigit()
               for pre in ("eri_", "eri32_", "grad_", "grad32_"))


def _flags(src):
    """nvcc flags of one source.  The generated class files are built
    without -lineinfo: their line tables (a line per recurrence term) double
    their objects, and the library with them would pass 400 MB.  Every
    hand-written source keeps -lineinfo."""
    if _generated_class(src):
        return [f for f in FLAGS if f != "-lineinfo"]
    return FLAGS


_INC = re.compile(r'^\s*#\s*include\s+"([^"]+)"', re.M)


def _deps(src, seen=None):
    """The file and every header it includes with quotes, recursively."""
    seen = set() if seen is None else seen
    if src in seen:
        return seen
    seen.add(src)
    with open(src) as fh:
        text = fh.read()
    for inc in _INC.findall(text):
        for base in (os.path.dirname(src), CSRC, GEN, os.path.join(HERE, "..", "include")):
            cand = os.path.normpath(os.path.join(base, inc))
            if os.path.exists(cand):
                _deps(cand, seen)
                break
    return seen


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(lmax=2, jobs=None, verbose=False):
    jobs = jobs or max(2, os.cpu_count() or 2)
    subprocess.run([sys.executable, os.path.join(CSRC, "gen_eri.py"), GEN, "--lmax", str(lmax)],
                   check=True, stdout=subprocess.DEVNULL)
    subprocess.run([sys.executable, os.path.join(CSRC, "gen_xc.py"), GEN], check=True, stdout=subprocess.DEVNULL)
    os.makedirs(OBJ, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith(".cu")]
    srcs += [os.path.join(CSRC, "xc", f) for f in sorted(os.listdir(os.path.join(CSRC, "xc"))) if f.endswith(".cu")]
    srcs += [os.path.join(GEN, f) for f in sorted(os.listdir(GEN)) if f.endswith(".cu")]
    # drop generated classes beyond lmax (left over from an earlier build)
    keep = []
    for s in srcs:
        b = os.path.basename(s)
        for pre in ("eri_", "eri32_", "grad_", "grad32_"):
            if b.startswith(pre) and b[len(pre):len(pre) + 4].isdigit():
                ls = [int(ch) for ch in b[len(pre):len(pre) + 4]]
                # classes up to lmax, plus the f classes with L sum <= F_MAX_L
                if max(ls) > lmax and sum(ls) > F_MAX_L:
                    break
        else:
            keep.append(s)
    srcs = keep
    objs = []
    todo = []
    for s in srcs:
        o = os.path.join(OBJ, os.path.basename(s)[:-3] + ".o")
        objs.append(o)
        if _newer(o, sorted(_deps(s))):
            todo.append((s, o))

    def cc(so):
        s, o = so
        cmd = [NVCC] + ARCH + _flags(s) + _extra_flags(s) + ["-c", s, "-o", o]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed on %s:\n%s" % (s, r.stderr[-4000:]))
        if verbose and r.stderr.strip():
            print(r.stderr)
        return o

    # longest compiles first
    todo.sort(key=lambda so: -os.path.getsize(so[0]))
    with ThreadPoolExecutor(jobs) as ex:
        list(ex.map(cc, todo))
    if todo or not os.path.exists(LIB):
        cmd = [NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-cudart", "static", "-lpthread"]
        subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--lmax", type=int, default=2)
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("-v", action="store_true")
    a = ap.parse_args()
    print(build(a.lmax, a.jobs, a.v))
