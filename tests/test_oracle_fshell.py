"""f shells (cc-pVTZ water): the oracle against QUICK's own CUDA_SPDF kernels
compiled for the host (oracle/build_ref.py --spdf / --accurate-boys).

Two defects of QUICK decide what can be compared:

* QUICK's Boys function FmT recurs upward from F_0 for every T > 3e-5 and
  loses most digits at small T and high m (checked below against the
  confluent hypergeometric function).  cc-pVTZ puts d shells on H, so
  quartets on one O-H bond reach high m at small T and QUICK's Fock matrix
  is off by up to 5e-4 there.  The `--accurate-boys` build is QUICK with
  only FmT replaced; against it the oracle agrees to 1e-13 on every Fock
  element that QUICK's spd kernels and its f zones for pairs with
  L_A + L_B <= 4 produce.
* QUICK's f zones for pairs with L_A + L_B = 5 or 6 (fd, ff) are not
  rotationally covariant: rotating the molecule by 90 degrees and the
  density with it changes QUICK's Fock matrix by O(1) (the oracle: 1e-14).
  Those elements are therefore compared with the oracle only, which the GPU
  matches (tests/test_gpu_fshell.py)."""
import copy

import numpy as np
import pytest

import oracle
from quick_b200.basis import build_basis
from quick_b200.molecule import water_cluster

HAVE_BOYS = oracle.ref_available("boys")
HAVE_SPDF = oracle.ref_available(True)


def _water(grid=(1, 1, 1)):
    m = water_cluster(grid, seed=0)
    return m, build_basis(m.symbols, "cc-pVTZ")


@pytest.mark.skipif(not oracle.ref_available(), reason="QUICK host build not present")
def test_quick_fmt_loses_accuracy_at_small_T():
    import ctypes as C
    from scipy.special import hyp1f1
    r = oracle.ref_lib()
    out = np.zeros(20)
    errs = {}
    for T in (1e-2, 1.0):
        r.qref_fmt(C.c_int(8), C.c_double(T), out.ctypes.data_as(C.c_void_p))
        ref = hyp1f1(6.5, 7.5, -T) / 13.0
        errs[T] = abs(out[6] - ref) / ref
    assert errs[1.0] < 1e-9          # fine at moderate T
    assert errs[1e-2] > 1e-2         # F_6(0.01) wrong in the second digit
    ours = oracle.boys(8, 1e-2)
    assert abs(ours[6] - hyp1f1(6.5, 7.5, -1e-2) / 13.0) < 1e-15


@pytest.mark.skipif(not HAVE_BOYS, reason="QUICK accurate-Boys host build not present")
@pytest.mark.parametrize("grid", [(1, 1, 1), (2, 1, 1)])
def test_oracle_matches_quick_spdf_on_pairs_up_to_l4(grid):
    """Coulomb from density on pairs with L_k + L_l <= 4, and full HF exchange
    from density on s and p functions, compared on Fock elements whose pair
    has L_i + L_j <= 4."""
    m, b = _water(grid)
    n = b.nbasis
    L = b.itype.sum(axis=0)
    Y, cp = oracle.schwarz(b, m.xyz_bohr)
    Z = np.zeros((n, n), order="F")
    low = (L[:, None] + L[None, :]) <= 4
    rng = np.random.default_rng(1)
    oracle.ref_upload_molecule(m, b, Y, cp, threads=8, spdf="boys")
    for method, mask in ((2, low), (0, np.outer(L <= 1, L <= 1))):
        D = rng.standard_normal((n, n)) * mask
        D = np.asfortranarray(D + D.T)
        cm = oracle.cutmatrix(b, D)
        ref = oracle.ref_get2e(Z, D, cm, 1e-12, 1e-20, method=method, spdf="boys")
        got, _ = oracle.fock(b, m.xyz_bohr, Y, cp, cm, D, 1e-12, 1e-20, hybrid={0: 1.0, 2: 0.0}[method], O=Z)
        assert np.abs((got - ref) * low).max() < 1e-10


def _rotation_error(fock_fn, m, b, D):
    """|T F(R, D) T^T - F(R', T D T^T)| for a 90 degree rotation about y,
    T the signed permutation of Cartesian components it induces."""
    n = b.nbasis
    m2 = copy.deepcopy(m)
    xa = m.xyz_angstrom
    m2.xyz_angstrom = np.stack([xa[:, 2], xa[:, 1], -xa[:, 0]], axis=1)
    T = np.zeros((n, n))
    for f in range(n):
        a, bb, c = (int(v) for v in b.itype[:, f])
        for g in range(n):
            if (b.ncenter[g] == b.ncenter[f] and abs(g - f) < 10 and np.allclose(b.aexp[:, g], b.aexp[:, f])
                    and tuple(int(v) for v in b.itype[:, g]) == (c, bb, a)):
                T[g, f] = (-1.0) ** a
                break
    assert np.allclose(np.abs(T).sum(axis=0), 1.0)
    F1 = fock_fn(m, D)
    F2 = fock_fn(m2, np.asfortranarray(T @ D @ T.T))
    return np.abs(T @ F1 @ T.T - F2).max()


def test_oracle_is_rotationally_covariant_with_f_shells():
    m, b = _water()
    rng = np.random.default_rng(3)
    D = rng.standard_normal((b.nbasis, b.nbasis)) * 0.1
    D = np.asfortranarray(D + D.T)
    Z = np.zeros_like(D)

    def fock(mol, Dm):
        Y, cp = oracle.schwarz(b, mol.xyz_bohr)
        return oracle.fock(b, mol.xyz_bohr, Y, cp, oracle.cutmatrix(b, Dm), Dm, 1e-12, 1e-20, O=Z)[0]
    assert _rotation_error(fock, m, b, D) < 1e-12


@pytest.mark.skipif(not HAVE_BOYS, reason="QUICK accurate-Boys host build not present")
def test_quick_fd_ff_zones_are_not_rotationally_covariant():
    """The evidence for comparing the fd/ff pairs with the oracle only."""
    m, b = _water()
    rng = np.random.default_rng(3)
    D = rng.standard_normal((b.nbasis, b.nbasis)) * 0.1
    D = np.asfortranarray(D + D.T)
    Z = np.zeros_like(D)

    def fock(mol, Dm):
        Y, cp = oracle.schwarz(b, mol.xyz_bohr)
        oracle.ref_upload_molecule(mol, b, Y, cp, threads=8, spdf="boys")
        return oracle.ref_get2e(Z, Dm, oracle.cutmatrix(b, Dm), 1e-12, 1e-20, spdf="boys")
    assert _rotation_error(fock, m, b, D) > 1e-2


def test_oracle_fshell_gradient_matches_finite_differences(oracle_lib):
    """The oracle's two-electron gradient with f shells (cc-pVTZ water)
    against central differences (h = 1e-4 bohr) of E2 = Tr[D G(D)]/2 with the
    density held fixed: the reference the GPU's f-class gradient is held to."""
    from tests.helpers import random_density
    m = water_cluster((1, 1, 1), seed=0)
    b = build_basis(m.symbols, "cc-pVTZ")
    D = random_density(b.nbasis, seed=5, scale=0.05)
    cut, plim = 1e-14, 1e-30
    X = m.xyz_bohr.copy()
    Y, cp = oracle_lib.schwarz(b, X)
    cm = oracle_lib.cutmatrix(b, D)
    g = oracle_lib.grad2e(b, X, Y, cp, cm, D, cut, plim)
    h = 1e-4
    for k in (0, 4, 8):
        xs = []
        for sgn in (1, -1):
            v = X.ravel(order="F").copy()
            v[k] += sgn * h
            Xd = np.asfortranarray(v.reshape(3, -1, order="F"))
            Yd, cpd = oracle_lib.schwarz(b, Xd)
            xs.append(oracle_lib.energy2e(b, Xd, Yd, cpd, cm, D, cut, plim))
        assert abs((xs[0] - xs[1]) / (2 * h) - g[k]) < 1e-6
