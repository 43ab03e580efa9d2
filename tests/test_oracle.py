"""The CPU oracle: Boys function, and parity with QUICK's own kernels
(golden fixtures made by tests/golden/make_golden.py from QUICK's CUDA
sources compiled as host code; the live comparison runs where that build is
present)."""
import os

import numpy as np
import pytest
from scipy.special import hyp1f1

from tests.helpers import case, random_density

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
FIXTURES = ["water2_631gs", "water3_631gss", "propane_631gss"]


@pytest.mark.parametrize("T", [0.0, 1e-9, 1e-4, 0.3, 2.9, 11.0, 34.9, 35.1, 80.0, 400.0])
def test_boys_against_hypergeometric(oracle_lib, T):
    F = oracle_lib.boys(12, T)
    for m in range(13):
        ref = hyp1f1(m + 0.5, m + 1.5, -T) / (2 * m + 1)
        assert abs(F[m] - ref) <= 5e-14 * ref + 1e-300


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_fock_matches_quick_golden(oracle_lib, name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    m, b = case(name)
    for method, h in ((0, 1.0), (1, 0.2)):
        got, _ = oracle_lib.fock(b, m.xyz_bohr, z["YCutoff"], z["cutPrim"], z["cutMatrix"], z["dense"],
                                 1e-10, 1e-20, hybrid=h, O=z["O_in"])
        assert np.abs(got - z["fock_m%d" % method]).max() < 1e-8


@pytest.mark.parametrize("name", FIXTURES)
def test_schwarz_inputs_stable(oracle_lib, name):
    """The fixtures' Schwarz bounds are the oracle's restatement of schwarz.f90."""
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    m, b = case(name)
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    assert np.allclose(Y, z["YCutoff"], rtol=1e-13, atol=0)
    assert np.allclose(cp, z["cutPrim"], rtol=1e-13, atol=0)


def test_schwarz_bounds_integrals(oracle_lib):
    """|(ab|cd)| <= Y(ab) Y(cd) on a sample of shell quartets."""
    m, b = case("water2_631gs")
    Y, _ = oracle_lib.schwarz(b, m.xyz_bohr)
    rng = np.random.default_rng(0)
    for _ in range(40):
        sh = rng.integers(0, b.nshell, 4)
        Ls = [int(b.Qstart[s]) for s in sh]
        blk = oracle_lib.shell_quartet(b, m.xyz_bohr, *[int(s) for s in sh], *Ls)
        assert np.abs(blk).max() <= Y[sh[0], sh[1]] * Y[sh[2], sh[3]] * (1 + 1e-12)


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="QUICK host build not present")
def test_oracle_matches_quick_live(oracle_lib):
    m, b = case("hexane_631gs")
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    D = random_density(b.nbasis, seed=3)
    cm = oracle_lib.cutmatrix(b, D)
    oracle_lib.ref_upload_molecule(m, b, Y, cp, threads=8)
    ref = oracle_lib.ref_get2e(np.zeros_like(D), D, cm, 1e-9, 1e-12)
    got, _ = oracle_lib.fock(b, m.xyz_bohr, Y, cp, cm, D, 1e-9, 1e-12)
    assert np.abs(got - ref).max() < 1e-8


def test_oracle_grad_matches_finite_differences(oracle_lib):
    """Analytic two-electron gradient vs central differences (h = 1e-4 bohr)
    of E2 = Tr[D G(D)]/2 with the density held fixed."""
    m, b = case("water2_631gs")
    D = random_density(b.nbasis, seed=3, scale=0.05)
    cut, plim = 1e-14, 1e-30
    X = m.xyz_bohr.copy()
    Y, cp = oracle_lib.schwarz(b, X)
    cm = oracle_lib.cutmatrix(b, D)
    g = oracle_lib.grad2e(b, X, Y, cp, cm, D, cut, plim)
    h = 1e-4
    for k in (0, 4, 8, 13):
        xs = []
        for sgn in (1, -1):
            v = X.ravel(order="F").copy()
            v[k] += sgn * h
            Xd = np.asfortranarray(v.reshape(3, -1, order="F"))
            Yd, cpd = oracle_lib.schwarz(b, Xd)
            xs.append(oracle_lib.energy2e(b, Xd, Yd, cpd, cm, D, cut, plim))
        assert abs((xs[0] - xs[1]) / (2 * h) - g[k]) < 1e-7


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="QUICK host build not present")
@pytest.mark.parametrize("name", ["water2_631gs", "propane_631gss"])
def test_oracle_grad_matches_quick_live(oracle_lib, name):
    m, b = case(name)
    D = random_density(b.nbasis, seed=3, scale=0.05)
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    cm = oracle_lib.cutmatrix(b, D)
    g = oracle_lib.grad2e(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20)
    oracle_lib.ref_upload_molecule(m, b, Y, cp, threads=8)
    gr = oracle_lib.ref_grad(np.zeros_like(g), D, cm, 1e-10, 1e-20)
    assert np.abs(g - gr).max() < 1e-8


@pytest.mark.parametrize("name", FIXTURES)
def test_oracle_grad_matches_quick_golden(oracle_lib, name):
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    m, b = case(name)
    g = oracle_lib.grad2e(b, m.xyz_bohr, z["YCutoff"], z["cutPrim"], z["grad_cutMatrix"], z["grad_dense"],
                          1e-10, 1e-20)
    assert np.abs(g - z["grad2e"]).max() < 1e-8
