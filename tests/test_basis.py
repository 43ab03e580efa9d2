"""QUICK basis arrays restated from src/basis.f90 (no GPU)."""
import numpy as np
import pytest

from quick_b200.basis import build_basis, xnorm
from quick_b200.molecule import linear_alkane, water_cluster


@pytest.mark.parametrize("grid,basis,nbasis,nshell,nprim", [
    ((2, 2, 1), "6-31G*", 76, 32, 76),          # (H2O)4 / 6-31G*
    ((4, 4, 2), "6-31G**", 800, 320, 672),      # (H2O)32 / 6-31G**
    ((4, 4, 2), "cc-pVTZ", 2080, 704, 1280),    # (H2O)32 / cc-pVTZ (Cartesian)
])
def test_workload_sizes(grid, basis, nbasis, nshell, nprim):
    m = water_cluster(grid, seed=0)
    b = build_basis(m.symbols, basis)
    assert (b.nbasis, b.nshell, b.nprim) == (nbasis, nshell, nprim)


def test_alkane_size():
    m = linear_alkane(40, seed=0)
    assert m.natom == 122
    b = build_basis(m.symbols, "6-31G**")
    assert b.nbasis == 1010
    x = m.xyz_angstrom
    d = np.linalg.norm(x[:, None] - x[None], axis=-1) + 9 * np.eye(len(x))
    assert d.min() > 1.0


def test_layout_invariants():
    m = water_cluster((2, 1, 1), seed=1)
    b = build_basis(m.symbols, "6-31G**")
    assert b.Ksumtype[0] == 1 and b.Ksumtype[-1] == b.nbasis + 1
    assert np.all(np.diff(b.Ksumtype) == b.ktype)
    assert np.all(np.diff(b.kstart) == b.kprim[:-1])
    # d components: QUICK order and cons (src/basis.f90:546-573)
    s = int(np.where(b.Qstart == 2)[0][0])
    f0 = b.Ksumtype[s] - 1
    assert [tuple(b.KLMN[:, f0 + k]) for k in range(6)] == [(2, 0, 0), (1, 1, 0), (0, 2, 0), (1, 0, 1), (0, 1, 1), (0, 0, 2)]
    assert np.allclose(b.cons[f0:f0 + 6], [1, 3 ** 0.5, 1, 3 ** 0.5, 3 ** 0.5, 1])


def test_contracted_s_is_normalised():
    """xnewnorm makes <s|s> = 1 for a contracted s shell."""
    m = water_cluster((1, 1, 1), seed=0)
    b = build_basis(m.symbols, "6-31G*")
    c = b.gccoeff[:6, 0]
    a = b.gcexpo[:6, 0]
    S = sum(c[i] * c[j] * (np.pi / (a[i] + a[j])) ** 1.5 for i in range(6) for j in range(6))
    assert abs(S - 1.0) < 1e-12


def test_xnorm_matches_closed_form():
    a = 0.8
    for (i, j, k) in [(0, 0, 0), (1, 0, 0), (2, 0, 0), (1, 1, 0)]:
        # N^2 * integral of x^2i y^2j z^2k exp(-2 a r^2) = 1
        from math import gamma, pi
        integ = 1.0
        for n in (i, j, k):
            integ *= gamma(n + 0.5) / (2 * a) ** (n + 0.5)
        assert abs(xnorm(a, i, j, k) ** 2 * integ - 1.0) < 1e-12
