"""The timed workloads against QUICK's own kernels.

(H2O)4 in 6-31G* (76 functions) and (H2O)32 in 6-31G** (800 functions, the
Fock-build benchmark), seeded clusters, the bench's model density: the GPU's
Fock matrix, two-electron gradient and shell-quartet count against QUICK's
get2e and gradient kernels compiled for the host (fixtures written by
tests/golden/make_config_golden.py from oracle/_ref/libquickref.so).

Tolerances: Fock elements 1e-8 (for the 800-function matrix on 20000 sampled
elements and the diagonal; the projections G R within the bound that an
element error of 1e-8 implies, 1e-8 sum_j |R_jk|); gradient 1e-8 Eh/bohr;
the unique shell-quartet count (the numerator of the quartets/s metric)
exactly equal to the count of QUICK's own walk.
"""
import os

import numpy as np
import pytest

from quick_b200.basis import build_basis
from quick_b200.molecule import model_density, water_cluster
from quick_b200.scf import shell_cut_matrix

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_F, TOL_G = 1e-8, 1e-8
CONFIGS = {0: ("config0_water4_631gs.npz", (2, 2, 1), "6-31G*"),
           1: ("config1_water32_631gss.npz", (4, 4, 2), "6-31G**")}


@pytest.fixture(scope="module")
def session():
    from quick_b200 import capi
    s = capi.Session(0)
    yield s
    s.close()


def _probes(n):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_config_golden", os.path.join(GOLDEN, "make_config_golden.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod.probes(n)


@pytest.mark.parametrize("k", sorted(CONFIGS))
def test_config_matches_quick(session, oracle_lib, k):
    fname, grid, basis = CONFIGS[k]
    z = np.load(os.path.join(GOLDEN, fname))
    m = water_cluster(grid, seed=0)
    b = build_basis(m.symbols, basis)
    n = b.nbasis
    assert n == int(z["nbasis"])
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    D = model_density(m, b, seed=0)
    cm = shell_cut_matrix(b, D)
    G = session.get2e(np.zeros((n, n), order="F"), D, cm, 1e-10, 1e-20, method=0)
    # the metric's numerator: QUICK's walk, once per unordered pair of pairs
    assert session.fock_stats()["quartets"] == int(z["unique_quartets"])
    if "G" in z.files:
        assert np.abs(G - z["G"]).max() < TOL_F
    else:
        R, idx = _probes(n)
        assert np.abs(G[idx[:, 0], idx[:, 1]] - z["sample"]).max() < TOL_F
        assert np.abs(np.diag(G) - z["diag"]).max() < TOL_F
        bound = TOL_F * np.abs(R).sum(axis=0)
        assert np.all(np.abs(G @ R - z["GR"]).max(axis=0) < bound)
    g = session.grad(np.zeros(3 * m.natom), D, cm, 1e-10, 1e-20)
    assert np.abs(g - z["grad"]).max() < TOL_G

