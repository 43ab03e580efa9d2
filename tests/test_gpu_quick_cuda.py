"""This build's Fock matrix and XC quadrature against QUICK's own CUDA run
on the same GPU.

QUICK's src/cuda/gpu.cu, gpu_type.cu, gpu_get2e.cu and gpu_getxc.cu, built
unchanged by nvcc for sm_100a with QUICK's flags and configuration
(oracle/_ref/gpu/libquickref.so, written by ``oracle/build_ref.py --gpu``),
driven through QUICK's gpu_init_ / gpu_upload_* / gpu_get2e_ sequence in a
child process (QUICK's library never shares a process with this package's),
on (H2O)4 in 6-31G* and on the (H2O)32 6-31G** workload of the Fock-build
benchmark, with the benchmark's model density; and QUICK's gpu_getxc_ (B3LYP,
SG1 grid) on (H2O)32 and C40H82 in 6-31G**.

Tolerance: 1e-8 Eh on every element of the 800 x 800 matrix (QUICK adds its
integrals in 1e-16 fixed point with fast-math exponentials, this build in
FP64).
"""
import os
import subprocess
import sys
import tempfile

import numpy as np
import pytest

from quick_b200.basis import build_basis
from quick_b200.molecule import model_density, water_cluster
from quick_b200.scf import shell_cut_matrix

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
QUICK_GPU = os.path.join(ROOT, "oracle", "_ref", "gpu", "libquickref.so")
TOL_F = 1e-8

CHILD = r"""
import sys
import numpy as np
sys.path.insert(0, sys.argv[1])
import oracle
from quick_b200.basis import build_basis, sigrad2
from quick_b200.molecule import linear_alkane, model_density, water_cluster
from quick_b200.scf import shell_cut_matrix
mol, basis, mode, out = sys.argv[2], sys.argv[3], sys.argv[4], sys.argv[5]
kind, arg = mol.split(":")
m = water_cluster(tuple(int(x) for x in arg.split(",")), seed=0) if kind == "water" else linear_alkane(int(arg), seed=1)
b = build_basis(m.symbols, basis)
Y, cp = oracle.schwarz(b, m.xyz_bohr)
keep = oracle.ref_upload_molecule(m, b, Y, cp, spdf="gpu", device=0)
if mode == "fock":
    D = model_density(m, b, seed=0)
    cm = shell_cut_matrix(b, D)
    Os = []
    for _ in range(2):
        O, wall, kern = oracle.ref_get2e_gpu_timed(np.zeros_like(D), D, cm, 1e-10, 1e-20)
        Os.append(O)
    np.savez(out, O=Os[-1], O0=Os[0], kernel_ms=kern)
else:
    D = np.load(out + ".in.npy")
    O, exc, nel, wall = oracle.ref_getxc_gpu_timed(D, sigrad2(b), method=1)
    np.savez(out, O=O, exc=exc, nel=nel, wall=wall)
"""


@pytest.fixture(scope="module")
def session():
    from quick_b200 import capi
    s = capi.Session(0)
    yield s
    s.close()


def quick_gpu(mol, basis, mode, dense=None):
    """QUICK's GPU build on molecule ``mol`` ("water:4,4,2" or "alkane:40")
    in a child process: mode "fock" (two builds) or "xc" (one B3LYP SG1
    quadrature of ``dense``).  Returns the child's arrays."""
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "o.npz")
        if dense is not None:
            np.save(out + ".in.npy", dense)
        p = subprocess.run([sys.executable, "-c", CHILD, ROOT, mol, basis, mode, out],
                           capture_output=True, text=True, timeout=900)
        assert p.returncode == 0, p.stderr[-2000:]
        z = np.load(out)
        return {k: z[k] for k in z.files}


def quick_gpu_fock(grid, basis):
    z = quick_gpu("water:" + ",".join(map(str, grid)), basis, "fock")
    return z["O"], z["O0"]


@pytest.mark.skipif(not os.path.exists(QUICK_GPU), reason="QUICK's GPU build (oracle/build_ref.py --gpu) absent")
@pytest.mark.parametrize("grid,basis", [((2, 2, 1), "6-31G*"), ((4, 4, 2), "6-31G**")])
def test_fock_matches_quick_cuda(session, oracle_lib, grid, basis):
    Oq, Oq0 = quick_gpu_fock(grid, basis)
    # QUICK's integer accumulation: two runs of its kernel agree bit for bit
    assert np.array_equal(Oq, Oq0)
    m = water_cluster(grid, seed=0)
    b = build_basis(m.symbols, basis)
    n = b.nbasis
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    D = model_density(m, b, seed=0)
    cm = shell_cut_matrix(b, D)
    G = session.get2e(np.zeros((n, n), order="F"), D, cm, 1e-10, 1e-20, method=0)
    assert Oq.shape == (n, n)
    assert np.abs(G - Oq).max() < TOL_F


@pytest.mark.skipif(not os.path.exists(QUICK_GPU), reason="QUICK's GPU build (oracle/build_ref.py --gpu) absent")
@pytest.mark.parametrize("mol", ["water:4,4,2", "alkane:40"])
def test_xc_matches_quick_cuda(session, oracle_lib, mol):
    """B3LYP on QUICK's SG1 grid, 6-31G**: (H2O)32 (the XC line of the
    benchmark, 800 functions) and C40H82 (1010 functions).  Tolerances: the
    operator 1e-8 absolute, the XC energy and electron count 1e-9 relative
    (QUICK sums them in 1e-16 fixed point)."""
    from quick_b200.basis import sigrad2
    from quick_b200.molecule import linear_alkane
    kind, arg = mol.split(":")
    m = water_cluster(tuple(int(x) for x in arg.split(",")), seed=0) if kind == "water" else linear_alkane(int(arg), seed=1)
    b = build_basis(m.symbols, "6-31G**")
    n = b.nbasis
    rng = np.random.default_rng(0)
    C = rng.standard_normal((n, m.n_electrons // 2)) * 0.05
    D = np.asfortranarray(2.0 * C @ C.T)
    z = quick_gpu(mol, "6-31G**", "xc", dense=D)
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    o, e, a, _ = session.getxc(np.zeros((n, n), order="F"), D, sigrad2(b), method=1)
    assert np.abs(o - z["O"]).max() < 1e-8
    assert abs(e - float(z["exc"])) <= 1e-9 * abs(float(z["exc"]))
    assert abs(a - float(z["nel"])) <= 1e-9 * abs(float(z["nel"]))
