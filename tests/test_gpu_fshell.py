"""f shells (cc-pVTZ: d on H, f on O): every class with an f shell runs the
generic warp-per-quartet kernel (eri_generic.cu).  Fock matrices against the
oracle (itself pinned to QUICK's CUDA_SPDF kernels, tests/test_oracle_spdf.py)
at 1e-8; f shells have no gradient or Schwarz kernel and say so."""
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


def test_fshell_gradient_and_schwarz_report_missing_kernels(session, oracle_lib):
    from quick_b200 import capi
    m, b = _mol((1, 1, 1))
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    D = random_density(b.nbasis, seed=5, scale=0.05)
    cm = oracle_lib.cutmatrix(b, D)
    with pytest.raises(capi.QuickB200Error, match="f shells"):
        session.grad(np.zeros(3 * m.natom), D, cm, 1e-10, 1e-20)
    with pytest.raises(capi.QuickB200Error, match="f shells"):
        session.schwarz()
