"""Mixed-precision Fock builds and gradients (qb_set_mixed_precision):
quartets whose Y_ab Y_cd DNMax bound is below the cut run in FP32.  Checked
against the FP64 oracle: Fock elements within 1e-7 and the two-electron
energy E2 = 1/2 sum D G within 1e-6 Eh (the 1 micro-Hartree target) at cut
1e-3; the two-electron gradient within 1e-5 Eh/bohr (the gradient target) at
cut 1e-3, with both lists non-empty; cut 0 gives the FP64 gradient exactly."""
import numpy as np
import pytest

from tests.helpers import case, random_density

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def session():
    from quick_b200 import capi
    s = capi.Session(0)
    yield s
    s.set_mixed_precision(0.0)
    s.close()


@pytest.mark.parametrize("name", ["water4_631gs", "propane_631gss", "hexane_631gs"])
def test_mixed_fock_within_tolerance(session, oracle_lib, name):
    m, b = case(name)
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    D = random_density(b.nbasis, seed=7)
    cm = oracle_lib.cutmatrix(b, D)
    ref, _ = oracle_lib.fock(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20, hybrid=1.0, O=np.zeros_like(D))
    try:
        session.set_mixed_precision(1e-3)
        got = session.get2e(np.zeros_like(D), D, cm, 1e-10, 1e-20, method=0)
        split = session.fock_split()
    finally:
        session.set_mixed_precision(0.0)
    assert split["fp32"] > 0 and split["fp64"] > 0
    assert np.abs(got - ref).max() < 1e-7
    assert abs(0.5 * np.sum(D * (got - ref))) < 1e-6


@pytest.mark.parametrize("name", ["water3_631gss", "propane_631gss"])
def test_mixed_gradient_within_tolerance(session, oracle_lib, name):
    m, b = case(name)
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    D = random_density(b.nbasis, seed=5, scale=0.05)
    cm = oracle_lib.cutmatrix(b, D)
    ref = oracle_lib.grad2e(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20)
    g0 = session.grad(np.zeros(3 * m.natom), D, cm, 1e-10, 1e-20)
    try:
        session.set_mixed_precision(1e-3)
        g1 = session.grad(np.zeros(3 * m.natom), D, cm, 1e-10, 1e-20)
        session.set_mixed_precision(0.0)
        g2 = session.grad(np.zeros(3 * m.natom), D, cm, 1e-10, 1e-20)
    finally:
        session.set_mixed_precision(0.0)
    assert np.abs(g0 - ref).max() < 1e-8
    assert np.abs(g1 - ref).max() < 1e-5
    assert np.abs(g1 - g0).max() > 0.0          # the FP32 list was used
    assert np.abs(g2 - g0).max() < 1e-12        # cut 0: every quartet in FP64 again
