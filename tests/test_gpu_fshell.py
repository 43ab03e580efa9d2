"""f shells (cc-pVTZ: d on H, f on O): the f classes with total angular
momentum up to 8 run generated straight-line kernels (FP64 only above 6:
their FP32 lists of the mixed split run the FP64 kernels), the larger ones
the generic block-per-quartet kernels (eri_generic.cu).  Fock matrices and
the two-electron gradient against the oracle (itself pinned to QUICK's
CUDA_SPDF kernels where those are right and to finite differences,
tests/test_oracle_fshell.py) at 1e-8; Schwarz bounds for f pair types on the
GPU."""
import numpy as np
import pytest

from quick_b200.basis import build_basis
from quick_b200.molecule import water_cluster
from tests.helpers import random_density

pytestmark = pytest.mark.gpu
TOL = 1e-8


@pytest.fixture(scope="module")
def session():
    from quick_b200 import capi
    s = capi.Session(0)
    yield s
    s.set_mixed_precision(0.0)
    s.close()


def _mol(grid, seed=0):
    m = water_cluster(grid, seed=seed)
    return m, build_basis(m.symbols, "cc-pVTZ")


@pytest.mark.parametrize("grid,method", [((1, 1, 1), 0), ((2, 1, 1), 0), ((2, 1, 1), 1), ((3, 1, 1), 0)])
def test_fshell_fock_matches_oracle(session, oracle_lib, grid, method):
    m, b = _mol(grid)
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    D = random_density(b.nbasis, seed=7)
    cm = oracle_lib.cutmatrix(b, D)
    H = random_density(b.nbasis, seed=8, scale=0.3)
    hyb = {0: 1.0, 1: 0.2}[method]
    ref, _ = oracle_lib.fock(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20, hybrid=hyb, O=H)
    got = session.get2e(H, D, cm, 1e-10, 1e-20, method=method)
    assert np.abs(got - ref).max() < TOL
    assert np.array_equal(got, got.T)


def test_fshell_mixed_precision_list(session, oracle_lib):
    """f classes on the FP32 list of the mixed split still compute in FP64."""
    m, b = _mol((2, 1, 1))
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    D = random_density(b.nbasis, seed=7)
    cm = oracle_lib.cutmatrix(b, D)
    ref, _ = oracle_lib.fock(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20, hybrid=1.0)
    try:
        session.set_mixed_precision(1e-3)
        got = session.get2e(np.zeros_like(D), D, cm, 1e-10, 1e-20, method=0)
    finally:
        session.set_mixed_precision(0.0)
    assert np.abs(got - ref).max() < 1e-7


def test_fshell_schwarz_bounds_on_gpu(session, oracle_lib):
    """gpu_schwarz_ for pair types with an f shell runs the generic
    recurrence program; YCutoff and cutPrim as QUICK's schwarz.f90 defines
    them (the oracle's restatement).  The closed-form horizontal recurrence
    sums in another order than the oracle's, which costs up to 2e-10
    relative on the smallest d/f bounds (measured; 1e-12 elsewhere), so the
    tolerance is 1e-9 relative."""
    m, b = _mol((2, 1, 1))
    session.upload_molecule(m, b)            # Schwarz bounds from the GPU
    Yo, cpo = oracle_lib.schwarz(b, m.xyz_bohr)
    np.testing.assert_allclose(session.YCutoff, Yo, rtol=1e-9, atol=1e-300)
    # cutPrim of far-apart primitive pairs reaches 1e-160; such values screen
    # nothing and their last digits are noise in either code
    np.testing.assert_allclose(session.cutPrim, cpo, rtol=1e-9, atol=1e-30)


@pytest.mark.parametrize("grid", [(1, 1, 1), (2, 1, 1)])
def test_fshell_gradient_matches_oracle(session, oracle_lib, grid):
    """The f-class gradient kernels (straight-line up to total angular
    momentum 8, generic above) with the s/p/d classes against the oracle's
    two-electron gradient: 1e-8 Eh/bohr absolute on gradients of order 1e2."""
    m, b = _mol(grid)
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    D = random_density(b.nbasis, seed=5, scale=0.05)
    cm = oracle_lib.cutmatrix(b, D)
    session.get2e(np.zeros((b.nbasis, b.nbasis), order="F"), D, cm, 1e-10, 1e-20, method=0)
    got = session.grad(np.zeros(3 * m.natom), D, cm, 1e-10, 1e-20)
    ref = oracle_lib.grad2e(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20)
    assert np.abs(got - ref).max() < TOL


def test_fshell_mixed_gradient(session, oracle_lib):
    """The mixed split on the gradient with f shells: FP32 kernels for the
    classes up to total angular momentum 6, the FP64 kernels on the FP32
    lists of the f classes of 7 and 8, the generic kernel above; against the
    oracle's FP64 gradient at 1e-6 Eh/bohr (the FP32 quartets' bound is 1e-3
    Eh per quartet before the density)."""
    m, b = _mol((2, 1, 1))
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    D = random_density(b.nbasis, seed=5, scale=0.05)
    cm = oracle_lib.cutmatrix(b, D)
    ref = oracle_lib.grad2e(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20)
    try:
        session.set_mixed_precision(1e-3)
        session.get2e(np.zeros((b.nbasis, b.nbasis), order="F"), D, cm, 1e-10, 1e-20, method=0)
        got = session.grad(np.zeros(3 * m.natom), D, cm, 1e-10, 1e-20)
    finally:
        session.set_mixed_precision(0.0)
    assert np.abs(got - ref).max() < 1e-6
