"""GPU XC quadrature (gpu_getxc_) against QUICK's own getxc_kernel, run as
host code: stored golden fixtures (tests/golden/make_golden.py) and live
calls into oracle/_ref when it is built.

Tolerances: the functional values agree with QUICK's generated code to
rounding (rtol 1e-9; QUICK's BLYP density derivative cancels to ~1e-11);
the operator to 1e-8 absolute and the energy and electron count to 1e-9
relative (QUICK sums in 1e-16 fixed point over ~10^4-10^5 points in another
order)."""
import os

import numpy as np
import pytest

from tests.helpers import case, psd_density, random_density

pytestmark = pytest.mark.gpu
GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
OTOL = 1e-8
STOL = 1e-9


@pytest.fixture(scope="module")
def session():
    from quick_b200 import capi
    s = capi.Session(0)
    yield s
    s.close()


def test_functional_matches_quick(session):
    from quick_b200 import capi
    g = np.load(os.path.join(GOLD, "xc_functional.npz"))
    for method in (1, 2):
        f, fr, fs = capi.xc_functional(method, g["rho"], g["sigma"])
        ref = g["m%d" % method]
        for got, col in ((f, 0), (fr, 1), (fs, 2)):
            np.testing.assert_allclose(got, ref[:, col], rtol=1e-9, atol=0.0)


def _check(got, ref_o, ref_s):
    o, e, a, b = got
    assert np.abs(o - ref_o).max() < OTOL
    assert np.array_equal(o, o.T)
    for x, y in zip((e, a, b), ref_s):
        assert abs(x - y) <= STOL * abs(y), (x, y)


@pytest.mark.parametrize("name", ["water2_631gs", "water3_631gss", "propane_631gss"])
@pytest.mark.parametrize("method", [1, 2])
def test_getxc_matches_golden(session, name, method):
    g = np.load(os.path.join(GOLD, name + ".npz"))
    m, b = case(name)
    session.upload_molecule(m, b, g["YCutoff"], g["cutPrim"])
    got = session.getxc(g["xc_O_in"], g["xc_dense"], g["xc_sigrad2"], method=method)
    _check(got, g["xc_O_m%d" % method], g["xc_scalars_m%d" % method])


def test_getxc_matches_live_quick(session, oracle_lib):
    oracle = oracle_lib
    if not oracle.ref_available():
        pytest.skip("QUICK host build (oracle/_ref) not present")
    from quick_b200.basis import sigrad2
    m, b = case("hexane_631gs")
    Y, cp = oracle.schwarz(b, m.xyz_bohr)
    sg = sigrad2(b)
    D = psd_density(b.nbasis, m.n_electrons // 2, seed=21)
    H = random_density(b.nbasis, seed=22, scale=0.3)
    oracle.ref_upload_molecule(m, b, Y, cp)
    ref = oracle.ref_getxc(H, D, sg, method=1, Eelxc=1.5, aelec=0.25, belec=0.5)
    session.upload_molecule(m, b, Y, cp)
    got = session.getxc(H, D, sg, method=1, Eelxc=1.5, aelec=0.25, belec=0.5)
    _check(got, ref[0], ref[1:])


def test_grid_is_reused_and_calls_repeat(session):
    g = np.load(os.path.join(GOLD, "water2_631gs.npz"))
    m, b = case("water2_631gs")
    session.upload_molecule(m, b, g["YCutoff"], g["cutPrim"])
    r1 = session.getxc(g["xc_O_in"], g["xc_dense"], g["xc_sigrad2"], method=1)
    s1 = session.xc_stats()
    r2 = session.getxc(g["xc_O_in"], g["xc_dense"], g["xc_sigrad2"], method=1)
    s2 = session.xc_stats()
    assert s1["npts"] == s2["npts"] > 0 and s2["ms_grid"] == 0.0
    assert np.array_equal(r1[0], r2[0]) and r1[1:] == r2[1:]
    pts = session.xc_grid()
    assert pts.shape == (s1["npts"], 4) and (pts[:, 3] > 1e-9).all()


def test_getxc_rejects_sg0_and_hf(session):
    from quick_b200 import capi
    g = np.load(os.path.join(GOLD, "water2_631gs.npz"))
    m, b = case("water2_631gs")
    session.upload_molecule(m, b, g["YCutoff"], g["cutPrim"])
    with pytest.raises(capi.QuickB200Error, match="SG1"):
        session.getxc(g["xc_O_in"], g["xc_dense"], g["xc_sigrad2"], method=1, isg=0)
    with pytest.raises(capi.QuickB200Error, match="functional"):
        session.getxc(g["xc_O_in"], g["xc_dense"], g["xc_sigrad2"], method=0)
