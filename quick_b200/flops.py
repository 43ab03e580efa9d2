"""Algorithmic floating-point work of the Fock build, per angular class.

Counts come from the recurrences themselves (the dependency graph the
generator walks, with each multiply-add counted as 2), not from the compiled
kernels, so redundant work in a kernel never inflates them:

  per primitive quartet   vertical recurrence [e0|f0]^(m) (graph size),
                          Boys function F_0..F_L (7-term Taylor step 14,
                          exp ~20, downward recursion 4 per order, scaling
                          L+1), quartet set-up 30, contraction 1 per target;
  per shell quartet       horizontal recurrence (graph size) and the J/K
                          digestion, 2 flops for each of the 6 sums every
                          integral enters (12 per Cartesian integral).
"""
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))


def class_table():
    with open(os.path.join(HERE, "csrc", "gen", "class_flops.json")) as fh:
        return json.load(fh)


def per_prim(tag, st):
    L = sum(int(ch) for ch in tag)
    return st["vrr_flops"] + 14 + 20 + 4 * L + (L + 1) + 30 + st["targets"]


def per_quartet(tag, st, exchange=True):
    return st["hrr_flops"] + (12 if exchange else 4) * st["ncomp"]


def fock_flops(class_L, quartets, prim_quartets, exchange=True):
    """Total algorithmic flops for per-class quartet and primitive-quartet counts."""
    tab = class_table()
    tot = 0.0
    for L, nq, npq in zip(class_L, quartets, prim_quartets):
        tag = "%d%d%d%d" % tuple(L)
        st = tab[tag]
        tot += npq * per_prim(tag, st) + nq * per_quartet(tag, st, exchange)
    return tot
