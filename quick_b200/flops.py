"""Algorithmic floating-point work of the Fock build, per angular class.

Counts come from the recurrences themselves, not from the compiled kernels,
so redundant work in a kernel never inflates them; two tables are kept,
the dependency graph the generator walks (class_flops.json) and a count
from the recurrence definitions alone (definition_class), each with every
multiply-add counted as 2:

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


def _ncart(n):
    return (n + 1) * (n + 2) // 2


def _carts(n):
    return [(x, y, n - x - y) for x in range(n, -1, -1) for y in range(n - x, -1, -1)]


def definition_class(la, lb, lc, ld):
    """The same quantities as a class_flops.json entry, counted from the
    recurrence definitions as a plain (unscheduled) evaluation performs them,
    independently of the generator's dependency graph:

      vertical    Head-Gordon-Pople [e0|f0]^(m) for every |e| <= la + lb,
                  |f| <= lc + ld and every order m the recursion reaches
                  (the loop structure of a textbook evaluation: bra terms
                  PA x + WP y (3) plus n_i/(2p) (x - rho/p y) (5) where the
                  lowered index exists; ket terms QC x + WQ y (3), the
                  n_i/(2q) term (5) and the cross term e_i/(2(p+q)) z (3));
      horizontal  (a, b+1_i| = (a+1_i, b| + AB_i (a, b|, 2 flops for every
                  distinct intermediate, bra side for each kept ket
                  component, then the ket side for each final bra pair;
      targets     contracted [e0|f0], |e| in [la, la+lb], |f| in [lc, lc+ld].
    """
    Lab, Lcd = la + lb, lc + ld
    M = Lab + Lcd
    vrr = 0
    for n in range(1, Lab + 1):
        for e in _carts(n):
            i = 0 if e[0] else (1 if e[1] else 2)
            lowered2 = e[i] >= 2
            vrr += (M - n + 1) * (3 + (5 if lowered2 else 0))
    ecarts = [e for n in range(0, Lab + 1) for e in _carts(n)]
    for n in range(1, Lcd + 1):
        for f in _carts(n):
            i = 0 if f[0] else (1 if f[1] else 2)
            lowered2 = f[i] >= 2
            for e in ecarts:
                reps = M - n - sum(e) + 1
                if reps <= 0:
                    continue
                vrr += reps * (3 + (5 if lowered2 else 0) + (3 if e[i] > 0 else 0))
    ne_sel = sum(_ncart(n) for n in range(la, Lab + 1))
    nf_sel = sum(_ncart(n) for n in range(lc, Lcd + 1))
    hrr = 0
    for j in range(1, lb + 1):
        for k in range(la, la + lb - j + 1):
            hrr += 2 * _ncart(k) * _ncart(j) * nf_sel
    nab = _ncart(la) * _ncart(lb)
    for j in range(1, ld + 1):
        for k in range(lc, lc + ld - j + 1):
            hrr += 2 * _ncart(k) * _ncart(j) * nab
    return {"vrr_flops": vrr, "hrr_flops": hrr, "targets": ne_sel * nf_sel,
            "ncomp": _ncart(la) * _ncart(lb) * _ncart(lc) * _ncart(ld)}


def fock_flops(class_L, quartets, prim_quartets, exchange=True, table="generator"):
    """Total algorithmic flops for per-class quartet and primitive-quartet
    counts.  table: "generator" (the recurrence graph the kernels' generator
    walks, class_flops.json), "definition" (definition_class), or "min" (the
    smaller of the two per class: neither a scheduling choice of the
    generator nor the redundancy of a plain evaluation inflates it)."""
    tab = class_table()
    tot = 0.0
    for L, nq, npq in zip(class_L, quartets, prim_quartets):
        tag = "%d%d%d%d" % tuple(L)
        gen, dfn = tab[tag], definition_class(*(int(x) for x in L))
        cost = []
        for st in ((gen,) if table == "generator" else (dfn,) if table == "definition" else (gen, dfn)):
            cost.append(npq * per_prim(tag, st) + nq * per_quartet(tag, st, exchange))
        tot += min(cost)
    return tot
