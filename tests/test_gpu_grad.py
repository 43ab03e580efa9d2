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
