"""The definition-level FLOP count of quick_b200.flops (an independent check
on the generator's own table): hand-counted small classes, and the same
targets and Cartesian component counts as the generator's table for every
class it holds."""
import os

import pytest

from quick_b200 import flops


def test_small_classes_by_hand():
    # (ps|ss): three [p0|00]^(0) = PA F0 + WP F1, 3 flops each
    assert flops.definition_class(1, 0, 0, 0)["vrr_flops"] == 9
    # (ds|ss): [p0|00]^(0,1) 3 x 2 x 3 = 18; [d0|00]^(0) 6 x 3 + 5 for xx, yy, zz = 33
    assert flops.definition_class(2, 0, 0, 0)["vrr_flops"] == 51
    # (pp|ss): (p, p+1_i| from (d| and (p|, 9 intermediates x 2
    assert flops.definition_class(1, 1, 0, 0)["hrr_flops"] == 18
    d = flops.definition_class(2, 1, 1, 1)
    assert (d["targets"], d["ncomp"]) == (16 * 9, 6 * 3 * 3 * 3)


@pytest.mark.skipif(not os.path.exists(os.path.join(flops.HERE, "csrc", "gen", "class_flops.json")),
                    reason="generated class table absent (run the build)")
def test_same_targets_as_generator():
    tab = flops.class_table()
    for tag, st in tab.items():
        d = flops.definition_class(*(int(c) for c in tag))
        assert (d["targets"], d["ncomp"]) == (st["targets"], st["ncomp"]), tag
        assert d["vrr_flops"] > 0 or sum(int(c) for c in tag) == 0


def test_min_table_is_the_smaller():
    cl = [(1, 0, 0, 0), (2, 2, 2, 2)]
    nq, npq = [10, 10], [40, 40]
    lo = flops.fock_flops(cl, nq, npq, table="min")
    assert lo <= flops.fock_flops(cl, nq, npq, table="generator")
    assert lo <= flops.fock_flops(cl, nq, npq, table="definition")
