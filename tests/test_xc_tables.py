"""CPU checks of the XC grid's constant tables (quick_b200/csrc/gen_xc.py,
quick_b200/data/lebedev.json) and of the basis-side XC inputs."""
import itertools
import json
import math
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "quick_b200", "csrc"))
import gen_xc  # noqa: E402

DEGREE = {6: 3, 38: 9, 86: 11, 194: 17, 302: 29}


def expand(orbits):
    """Points of the Lebedev-Laikov octahedral orbits (codes 1-6)."""
    pts = []
    for code, a, b, v in orbits:
        if code == 1:
            base = [(1.0, 0.0, 0.0)]
        elif code == 2:
            s = math.sqrt(0.5)
            base = [(0.0, s, s)]
        elif code == 3:
            s = math.sqrt(1.0 / 3.0)
            base = [(s, s, s)]
        elif code == 4:
            base = [(a, a, math.sqrt(1.0 - 2.0 * a * a))]
        elif code == 5:
            base = [(a, math.sqrt(1.0 - a * a), 0.0)]
        else:
            base = [(a, b, math.sqrt(1.0 - a * a - b * b))]
        orbit = set()
        for p in base:
            for perm in itertools.permutations(p):
                for sg in itertools.product((1.0, -1.0), repeat=3):
                    orbit.add(tuple(round(s * c, 15) + 0.0 for s, c in zip(sg, perm)))
        pts += [(x, y, z, v) for (x, y, z) in sorted(orbit)]
    return np.array(pts)


def sphere_mean(a, b, c):
    """Mean of x^a y^b z^c over the unit sphere."""
    if a % 2 or b % 2 or c % 2:
        return 0.0
    df = lambda n: math.prod(range(n, 0, -2)) if n > 0 else 1  # noqa: E731
    return df(a - 1) * df(b - 1) * df(c - 1) / df(a + b + c + 1)


@pytest.mark.parametrize("order", [6, 38, 86, 194, 302])
def test_lebedev_exact_to_its_degree(order):
    with open(os.path.join(ROOT, "quick_b200", "data", "lebedev.json")) as fh:
        leb = json.load(fh)
    p = expand(leb[str(order)])
    assert len(p) == order
    np.testing.assert_allclose(np.linalg.norm(p[:, :3], axis=1), 1.0, atol=1e-15)
    assert abs(p[:, 3].sum() - 1.0) < 1e-14
    L = DEGREE[order]
    for a in range(L + 1):
        for b in range(L + 1 - a):
            for c in range(L + 1 - a - b):
                got = float((p[:, 3] * p[:, 0] ** a * p[:, 1] ** b * p[:, 2] ** c).sum())
                assert abs(got - sphere_mean(a, b, c)) < 1e-14, (order, a, b, c)


def test_radial_grid_is_euler_maclaurin():
    r, w = gen_xc.radial_grid()
    assert len(r) == len(w) == 50
    for i in range(1, 51):
        assert abs(r[i - 1] - i * i / (51 - i) ** 2) <= 5e-13 * max(1.0, r[i - 1])
        assert abs(w[i - 1] - 2 * 51 * i ** 5 / (51 - i) ** 7) <= 5e-13 * max(1.0, w[i - 1])
    # the grid integrates r^2 exp(-r^2) (in units of the atomic radius) accurately
    x, wt = np.array(r), np.array(w)
    assert abs((wt * np.exp(-x * x)).sum() - math.sqrt(math.pi) / 4.0) < 1e-6


def test_radial_grid_matches_quick_table():
    from oracle.build_ref import quick_root
    src = os.path.join(quick_root(), "src", "cuda", "gpu_getxc.cu")
    if not os.path.exists(src):
        pytest.skip("QUICK source tree not present")
    import re
    text = open(src).read()
    tab = lambda name: [float(x) for x in re.search(name + r"\[50\] = \{(.*?)\};", text, re.S).group(1)  # noqa: E731
                        .replace("\n", " ").split(",") if x.strip()]
    r, w = gen_xc.radial_grid()
    assert r == tab("RGRID")
    qw = tab("RWT")
    # QUICK's entry 48 was printed from a double one ulp below the exact value
    assert all(abs(a - b) <= 2e-16 * abs(b) for a, b in zip(w, qw))
    assert sum(a != b for a, b in zip(w, qw)) <= 1


def test_sigrad2_is_the_significance_radius():
    from quick_b200.basis import build_basis, sigrad2
    from quick_b200.molecule import water_cluster
    m = water_cluster((1, 1, 1), seed=0)
    b = build_basis(m.symbols, "6-31G**")
    s2 = sigrad2(b)
    for f in range(b.nbasis):
        amin = min(b.aexp[c, f] for c in range(b.ncontract[f]))
        L = int(b.itype[:, f].sum())
        g = math.gamma(L + 1.5) / math.sqrt(math.pi) * 11.13665599366341569
        target = 1e-10 * (((2 * amin) ** (L + 1.5)) / g) ** -0.5
        r = math.sqrt(s2[f])
        val = lambda x: math.exp(-amin * x * x) * x ** L  # noqa: E731
        assert val(r) >= target * (1 - 1e-12) and val(r + 1.0e-3) < target   # the search stops after its 1e-3 steps


def test_dcoeff_is_normalised():
    """Each contracted function has unit self-overlap after normalize_basis."""
    from quick_b200.basis import build_basis
    from quick_b200.molecule import water_cluster
    m = water_cluster((1, 1, 1), seed=0)
    b = build_basis(m.symbols, "6-31G*")
    for f in range(b.nbasis):
        i, j, k = (int(v) for v in b.itype[:, f])
        s = 0.0
        for c1 in range(b.ncontract[f]):
            for c2 in range(b.ncontract[f]):
                p = b.aexp[c1, f] + b.aexp[c2, f]
                dfac = 1.0
                for n in (i, j, k):
                    dfac *= math.prod(range(2 * n - 1, 0, -2)) if n else 1.0
                s += b.dcoeff[c1, f] * b.dcoeff[c2, f] * dfac * (math.pi / p) ** 1.5 / (2 * p) ** (i + j + k)
        assert abs(s - 1.0) < 1e-12, (f, s)


def test_xc_golden_fixtures_are_consistent():
    for name in ("water2_631gs", "water3_631gss", "propane_631gss"):
        g = np.load(os.path.join(ROOT, "tests", "golden", name + ".npz"))
        for m in (1, 2):
            e, a, b = g["xc_scalars_m%d" % m]
            assert a == b and a > 0 and e < 0
            o = g["xc_O_m%d" % m]
            assert np.array_equal(o, o.T)
