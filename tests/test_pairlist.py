"""QUICK's shell-pair list (gpu.cu:401-1003), bit-exact, built by this
package's host code without a GPU."""
import os

import numpy as np
import pytest

from tests.helpers import case

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")


@pytest.mark.parametrize("name", ["water2_631gs", "water3_631gss", "propane_631gss"])
def test_pairlist_matches_quick_golden(name):
    from quick_b200 import capi
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    m, b = case(name)
    got = capi.build_pairlist_host(b, z["YCutoff"])
    assert np.array_equal(got["pairs"], z["pairs"])
    assert got["fStart"] == int(z["fStart"]) and got["ffStart"] == int(z["ffStart"])
    assert np.array_equal(got["sorted_Q"], z["sorted_Q"])
    assert np.array_equal(got["sorted_Qnumber"], z["sorted_Qnumber"])


@pytest.mark.skipif(not __import__("oracle").ref_available(), reason="QUICK host build not present")
def test_pairlist_matches_quick_live_with_f_shells(oracle_lib):
    from quick_b200 import capi
    from quick_b200.basis import build_basis
    from quick_b200.molecule import water_cluster
    m = water_cluster((2, 1, 1), seed=5)
    b = build_basis(m.symbols, "cc-pVTZ")
    Y, cp = oracle_lib.schwarz(b, m.xyz_bohr)
    oracle_lib.ref_upload_molecule(m, b, Y, cp)
    ref = oracle_lib.ref_pairlist()
    got = capi.build_pairlist_host(b, Y)
    assert np.array_equal(got["pairs"], ref["pairs"])
    assert (got["fStart"], got["ffStart"]) == (ref["fStart"], ref["ffStart"])


def test_pairlist_ties_keep_insertion_order():
    """Equal keys stay in scan order, as QUICK's bubble sort leaves them."""
    from quick_b200 import capi
    from quick_b200.basis import build_basis
    from quick_b200.molecule import Molecule
    # two identical, far-apart H atoms: many exactly equal Schwarz bounds
    m = Molecule(["H", "H", "H"], np.array([[0.0, 0, 0], [0, 0, 5.0], [0, 0, 10.0]]))
    b = build_basis(m.symbols, "6-31G*")
    Y = np.ones((b.nshell, b.nshell), order="F") * 1e-5
    got = capi.build_pairlist_host(b, Y)
    # Every bound is 1e-5 (band 2 of gpu.cu:532-636), so the Schwarz sort
    # leaves QUICK's scan order and only the stable primitive-count sort
    # (kprim(x) kprim(y) descending, then kprim(x) descending) reorders it.
    sq, sqn, kp = got["sorted_Q"], got["sorted_Qnumber"], b.kprim
    want = []
    for qp in range(7):
        for q in range(4):
            for p in range(4):
                if p + q != qp:
                    continue
                blk = [(i, j) for i in range(len(sq)) for j in range(len(sq))
                       if sqn[i] == q and sqn[j] == p and sq[i] <= sq[j]]
                blk.sort(key=lambda e: (-int(kp[sq[e[0]]]) * int(kp[sq[e[1]]]), -int(kp[sq[e[0]]])))
                want += blk
    xs = [tuple(int(v) for v in p) for p in got["pairs"]]
    assert len(xs) > 0 and xs == want
