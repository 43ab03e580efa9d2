"""This build's Fock matrix against QUICK's own CUDA run on the same GPU.

QUICK's src/cuda/gpu.cu, gpu_type.cu, gpu_get2e.cu and gpu_getxc.cu, built
unchanged by nvcc for sm_100a with QUICK's flags and configuration
(oracle/_ref/gpu/libquickref.so, written by ``oracle/build_ref.py --gpu``),
driven through QUICK's gpu_init_ / gpu_upload_* / gpu_get2e_ sequence in a
child process (QUICK's library never shares a process with this package's),
on (H2O)4 in 6-31G* and on the (H2O)32 6-31G** workload of the Fock-build
benchmark, with the benchmark's model density.

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
from quick_b200.basis import build_basis
from quick_b200.molecule import model_density, water_cluster
from quick_b200.scf import shell_cut_matrix
grid, basis, out = tuple(int(x) for x in sys.argv[2].split(",")), sys.argv[3], sys.argv[4]
m = water_cluster(grid, seed=0)
b = build_basis(m.symbols, basis)
Y, cp = oracle.schwarz(b, m.xyz_bohr)
keep = oracle.ref_upload_molecule(m, b, Y, cp, spdf="gpu", device=0)
D = model_density(m, b, seed=0)
cm = shell_cut_matrix(b, D)
Os = []
for _ in range(2):
    O, wall, kern = oracle.ref_get2e_gpu_timed(np.zeros_like(D), D, cm, 1e-10, 1e-20)
    Os.append(O)
np.savez(out, O=Os[-1], O0=Os[0], kernel_ms=kern)
"""


@pytest.fixture(scope="module")
def session():
    from quick_b200 import capi
    s = capi.Session(0)
    yield s
    s.close()


def quick_gpu_fock(grid, basis):
    with tempfile.TemporaryDirectory() as d:
        out = os.path.join(d, "o.npz")
        p = subprocess.run([sys.executable, "-c", CHILD, ROOT, ",".join(map(str, grid)), basis, out],
                           capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stderr[-2000:]
        z = np.load(out)
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
