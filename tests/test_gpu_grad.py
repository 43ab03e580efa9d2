"""GPU nuclear gradient of the two-electron energy against the CPU oracle,
which is pinned to central finite differences of the energy and to QUICK's
own gradient kernel (tests/test_oracle.py).  Tolerance 1e-8 Eh/bohr."""
import numpy as np
import pytest

from tests.helpers import CASES, case, random_density

pytestmark = pytest.mark.gpu
TOL = 1e-8


@pytest.fixture(scope="module")
def session():
    from quick_b200 import capi
    s = capi.Session(0)
    yield s
    s.close()


@pytest.mark.parametrize("name", sorted(CASES))
def test_grad_matches_oracle(session, oracle_lib, name):
    m, b = case(name)
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    D = random_density(b.nbasis, seed=5, scale=0.05)
    cm = oracle_lib.cutmatrix(b, D)
    g0 = np.random.default_rng(1).standard_normal(3 * m.natom)
    ref = g0 + oracle_lib.grad2e(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20)
    got = session.grad(g0, D, cm, 1e-10, 1e-20)
    assert np.abs(got - ref).max() < TOL, (name, np.abs(got - ref).max())
    # translational invariance of the two-electron part
    assert np.abs((got - g0).reshape(-1, 3).sum(axis=0)).max() < 1e-9


def test_autotuned_gradient_lanes_match_oracle(oracle_lib):
    """qb_autotune_grad times 1, 2 and 4 lanes per quartet for the light
    gradient classes on the last gradient's lists and keeps the fastest; the
    gradient with the chosen sizes still matches the oracle (1e-8), and the
    sizes are among the compiled ones."""
    from quick_b200 import capi
    m, b = case("water4_631gs")
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    s = capi.Session(0)
    try:
        s.upload_molecule(m, b, Y, cp)
        D = random_density(b.nbasis, seed=5, scale=0.05)
        cm = oracle_lib.cutmatrix(b, D)
        ref = oracle_lib.grad2e(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20)
        s.grad(np.zeros(3 * m.natom), D, cm, 1e-10, 1e-20)
        g = s.autotune_grad()
        got = s.grad(np.zeros(3 * m.natom), D, cm, 1e-10, 1e-20)
        # every compiled size forced in turn on the light classes
        forced = {}
        for lanes in (2, 4):
            s.set_grad_groups([lanes if sum_l <= 2 else 1 for sum_l in _class_l_sums()])
            forced[lanes] = s.grad(np.zeros(3 * m.natom), D, cm, 1e-10, 1e-20)
        with pytest.raises(capi.QuickB200Error):
            s.set_grad_groups([3] * len(_class_l_sums()))
    finally:
        s.close()
    assert set(int(x) for x in g if x) <= {1, 2, 4}
    assert np.abs(got - ref).max() < TOL
    for lanes, f in forced.items():
        assert np.abs(f - ref).max() < TOL, lanes


def _class_l_sums():
    """Total angular momentum of every class of the library's class table."""
    from quick_b200 import capi
    n_c = capi.C.c_int(0)
    cl = np.zeros(4 * 128, dtype=np.int32)
    cq = np.zeros(128, dtype=np.int64)
    capi.lib().qb_class_info(capi.C.byref(n_c), capi._ptr(cl), capi._ptr(cq), 128)
    return [int(cl[4 * i:4 * i + 4].sum()) for i in range(n_c.value)]
