"""GPU Fock build against the CPU oracle (which is itself pinned to QUICK's
own kernels by tests/test_oracle.py and the fixtures of tests/golden/).
Tolerance: 1e-8 on Fock elements."""
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
@pytest.mark.parametrize("method", [0, 1])
def test_fock_matches_oracle(session, oracle_lib, name, method):
    oracle = oracle_lib
    m, b = case(name)
    Y, cp = oracle.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    D = random_density(b.nbasis, seed=7)
    cm = oracle.cutmatrix(b, D)
    H = random_density(b.nbasis, seed=8, scale=0.3)
    hyb = {0: 1.0, 1: 0.2, 2: 0.0}[method]
    ref, cnt = oracle.fock(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20, hybrid=hyb, O=H)
    got = session.get2e(H, D, cm, 1e-10, 1e-20, method=method)
    err = np.abs(got - ref).max()
    assert err < TOL, (name, err)
    assert np.array_equal(got, got.T)


def test_pairlist_matches_host(session, oracle_lib):
    from quick_b200 import capi
    m, b = case("water3_631gss")
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    dev = session.pairlist()
    host = capi.build_pairlist_host(b, Y)
    assert np.array_equal(dev["pairs"], host["pairs"])
    assert (dev["fStart"], dev["ffStart"]) == (host["fStart"], host["ffStart"])


def test_repeated_builds_reuse_buffers(session, oracle_lib):
    m, b = case("water2_631gs")
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    for seed in range(3):
        D = random_density(b.nbasis, seed=seed)
        cm = oracle_lib.cutmatrix(b, D)
        ref, _ = oracle_lib.fock(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20)
        got = session.get2e(np.zeros_like(D), D, cm, 1e-10, 1e-20)
        assert np.abs(got - ref).max() < TOL


@pytest.mark.parametrize("name", ["water2_631gs", "propane_631gss"])
def test_schwarz_kernel_matches_oracle(session, oracle_lib, name):
    """YCutoff / cutPrim from the GPU kernel against the oracle's restatement
    of schwarz.f90 (relative 1e-12; cutPrim entries below 1e-150 skipped,
    their squares are subnormal)."""
    m, b = case(name)
    Yo, cpo = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b)          # GPU Schwarz path
    Y, cp = session.YCutoff, session.cutPrim
    assert np.all((Y > 0) == (Yo > 0))
    mask = Yo > 0
    assert np.max(np.abs(Y[mask] - Yo[mask]) / Yo[mask]) < 1e-12
    big = cpo > 1e-150
    assert np.array_equal(cp > 0, cpo > 0)
    assert np.max(np.abs(cp[big] - cpo[big]) / cpo[big]) < 1e-12


def test_autotuned_lane_groups_keep_the_fock_matrix():
    """qb_autotune_classes picks, per class, the fastest compiled lane-group
    size on the last build's quartet lists; the Fock matrix after tuning
    equals the one before (different summation order only: 1e-10)."""
    from quick_b200 import capi
    from quick_b200.molecule import water_cluster
    from quick_b200.basis import build_basis
    from quick_b200.scf import shell_cut_matrix
    m = water_cluster((2, 2, 1), seed=1)
    b = build_basis(m.symbols, "6-31G**")
    s = capi.Session(0)
    try:
        s.upload_molecule(m, b)
        D = random_density(b.nbasis, seed=2, scale=0.05)
        cm = shell_cut_matrix(b, D)
        O = np.zeros((b.nbasis, b.nbasis), order="F")
        F0 = s.get2e(O, D, cm, 1e-10, 1e-20)
        g = s.autotune()
        F1 = s.get2e(O, D, cm, 1e-10, 1e-20)
    finally:
        s.close()
    assert np.abs(F1 - F0).max() < 1e-10
    # lanes per quartet, or 256 + lanes for the staged-Boys kernels
    assert set(int(x) for x in g if x) <= {1, 2, 4, 8, 16, 32, 257, 258, 260}


@pytest.mark.parametrize("lanes", [1, 2, 4])
def test_staged_boys_kernels_match_oracle(oracle_lib, lanes):
    """The light classes' kernels that stage the Boys records in shared
    memory (variant 256 + lanes, forced with qb_set_class_groups) give the
    oracle's Fock matrix (1e-8), also with the mixed split on (FP32 lists in
    the plain FP32 kernels: within 1e-6)."""
    from quick_b200 import capi
    m, b = case("water4_631gs")
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    s = capi.Session(0)
    try:
        s.upload_molecule(m, b, Y, cp)
        D = random_density(b.nbasis, seed=7)
        cm = oracle_lib.cutmatrix(b, D)
        ref, _ = oracle_lib.fock(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20, hybrid=1.0)
        n_c = capi.C.c_int(0)
        cl = np.zeros(4 * 128, dtype=np.int32)
        cq = np.zeros(128, dtype=np.int64)
        capi.lib().qb_class_info(capi.C.byref(n_c), capi._ptr(cl), capi._ptr(cq), 128)
        ncls = n_c.value
        staged = []
        for fp32 in (False, True):
            codes = []
            for k in range(ncls):
                v = capi.Session.class_variants(k, fp32)
                codes.append(256 + lanes if 256 + lanes in v else v[0])
            staged.append(sum(c > 256 for c in codes))
            s.set_class_groups(codes, fp32=fp32)
        got = s.get2e(np.zeros((b.nbasis, b.nbasis), order="F"), D, cm, 1e-10, 1e-20, method=0)
        s.set_mixed_precision(1e-3)
        mixed = s.get2e(np.zeros((b.nbasis, b.nbasis), order="F"), D, cm, 1e-10, 1e-20, method=0)
        with pytest.raises(capi.QuickB200Error):
            s.set_class_groups([999] * ncls)
    finally:
        s.set_mixed_precision(0.0)
        s.close()
    assert staged[0] == 5 and staged[1] == 0    # ssss, psss, psps, ppss, dsss; no FP32 variant
    assert np.abs(got - ref).max() < TOL
    assert np.abs(mixed - ref).max() < 1e-6


def test_fixed_point_fock_is_bit_reproducible(oracle_lib):
    """qb_set_fixed_point(1): the Fock matrix is bit-identical over repeated
    builds (the screen lists the quartets in a different order each time and
    the atomics land in a different order), within 1e-12 of the FP64 build,
    and within 1e-13 after the lane groups change (a quartet's primitive sum
    then runs in another order); the FP64 build matches the oracle to 1e-8."""
    from quick_b200 import capi
    m, b = case("water4_631gs")
    n = b.nbasis
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    s = capi.Session(0)
    try:
        s.upload_molecule(m, b, Y, cp)
        D = random_density(n, seed=21)
        cm = oracle_lib.cutmatrix(b, D)
        f64 = s.get2e(np.zeros((n, n), order="F"), D, cm, 1e-10, 1e-20)
        capi.lib().qb_set_fixed_point(1)
        runs = [s.get2e(np.zeros((n, n), order="F"), D, cm, 1e-10, 1e-20) for _ in range(3)]
        s.autotune()
        runs.append(s.get2e(np.zeros((n, n), order="F"), D, cm, 1e-10, 1e-20))
    finally:
        capi.lib().qb_set_fixed_point(0)
        s.close()
    for r in runs[1:3]:
        assert np.array_equal(r, runs[0])
    assert np.abs(runs[3] - runs[0]).max() < 1e-13
    assert np.abs(runs[0] - f64).max() < 1e-12
    ref, _ = oracle_lib.fock(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20)
    assert np.abs(f64 - ref).max() < 1e-8


def test_fock_and_gradient_in_bra_range_passes(oracle_lib):
    """With a quartet-list budget far below the whole list (QB_LIST_BUDGET_MB
    = 0.25), the lists are written and consumed in passes over disjoint bra
    ranges; the Fock matrix, the gradient and the screened-quartet count
    equal the one-pass results (Fock and gradient to the oracle at 1e-8)."""
    import os
    from quick_b200 import capi
    m, b = case("water4_631gs")
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    D = random_density(b.nbasis, seed=7, scale=0.05)
    cm = oracle_lib.cutmatrix(b, D)
    ref, _ = oracle_lib.fock(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20, hybrid=1.0)
    gref = oracle_lib.grad2e(b, m.xyz_bohr, Y, cp, cm, D, 1e-10, 1e-20)
    out = {}
    for budget in (None, "0.25"):
        if budget:
            os.environ["QB_LIST_BUDGET_MB"] = budget
        s = capi.Session(0)
        try:
            s.upload_molecule(m, b, Y, cp)
            F = s.get2e(np.zeros((b.nbasis, b.nbasis), order="F"), D, cm, 1e-10, 1e-20, method=0)
            q = s.fock_stats()["quartets"]
            g = s.grad(np.zeros(3 * m.natom), D, cm, 1e-10, 1e-20)
            out[budget] = (F, q, g, capi.lib().qb_list_passes())
        finally:
            os.environ.pop("QB_LIST_BUDGET_MB", None)
            s.close()
    F1, q1, g1, p1 = out[None]
    Fp, qp, gp, pp = out["0.25"]
    assert p1 == 1 and pp > 1
    assert qp == q1
    assert np.abs(F1 - ref).max() < TOL and np.abs(Fp - ref).max() < TOL
    assert np.abs(g1 - gref).max() < TOL and np.abs(gp - gref).max() < TOL
