"""The f-shell workload's basis, cc-pVTZ, on (H2O)8 against the C oracle
(tests/golden/config4s_water8_ccpvtz.npz, written by
tests/golden/make_config_golden.py --only 4).  Kept in a file that pytest
collects after the other GPU Fock tests.

Tolerances as for the 800-function benchmark matrix: 1e-8 on 20000 sampled
elements and the diagonal, projections within the bound an element error of
1e-8 implies."""
import os

import numpy as np
import pytest

from quick_b200.basis import build_basis
from quick_b200.molecule import model_density, water_cluster
from quick_b200.scf import shell_cut_matrix

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
TOL_F = 1e-8


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


def test_fshell_workload_matches_oracle(session, oracle_lib):
    """The f-shell workload's basis, cc-pVTZ, on (H2O)8 (520 functions, the
    largest cluster the C oracle builds in about a minute; fixture written by
    make_config_golden.py --only 4): the GPU's Fock matrix against the
    oracle's on 20000 sampled elements, the diagonal and 8 projections
    (tolerances as for config 1)."""
    z = np.load(os.path.join(GOLDEN, "config4s_water8_ccpvtz.npz"))
    m = water_cluster((2, 2, 2), seed=0)
    b = build_basis(m.symbols, "cc-pVTZ")
    n = b.nbasis
    assert n == int(z["nbasis"])
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    session.upload_molecule(m, b, Y, cp)
    D = model_density(m, b, seed=0)
    cm = shell_cut_matrix(b, D)
    G = session.get2e(np.zeros((n, n), order="F"), D, cm, 1e-10, 1e-20, method=0)
    R, idx = _probes(n)
    assert np.abs(G[idx[:, 0], idx[:, 1]] - z["sample"]).max() < TOL_F
    assert np.abs(np.diag(G) - z["diag"]).max() < TOL_F
    bound = TOL_F * np.abs(R).sum(axis=0)
    assert np.all(np.abs(G @ R - z["GR"]).max(axis=0) < bound)
