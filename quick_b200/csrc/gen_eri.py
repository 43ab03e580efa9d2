"""Generate the per-class electron-repulsion kernels of the Fock build.

For every angular-momentum class (LA LB | LC LD) with LA >= LB, LC >= LD and
bra total >= ket total, this script writes straight-line CUDA for one shell
quartet per thread:

  * the Head-Gordon-Pople vertical recurrence (Obara-Saika form) producing
    [e0|f0]^(0) for LA <= |e| <= LA+LB, LC <= |f| <= LC+LD from F_m(T),
    emitted from a dependency walk so only intermediates that feed a target
    are computed;
  * contraction of those targets over the primitive quartets;
  * the horizontal recurrence (a,b+1_i| = (a+1_i,b| + AB_i (a,b| on both
    sides, with common sub-expressions shared;
  * the Coulomb/exchange digestion of the (ab|cd) block into the Fock
    matrix, bra-side Coulomb terms reduced across the warp first.

This is the same algorithm QUICK's generated int.h / gpu_get2e_subs_hrr.h
implement (gpu_get2e_subs.h:586-850), emitted by our own generator with
register-resident intermediates instead of QUICK's local-memory `store`.

Cartesian components of each shell are produced in QUICK's basis-function
order (src/basis.f90:546-643), so component k of a sub-shell is basis
function first+k.

    python gen_eri.py OUTDIR [--lmax 2]
"""
import itertools
import os
import sys

# QUICK's Cartesian order per shell (KLMN as readbasis assigns it)
QUICK_ORDER = {
    0: [(0, 0, 0)],
    1: [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
    2: [(2, 0, 0), (1, 1, 0), (0, 2, 0), (1, 0, 1), (0, 1, 1), (0, 0, 2)],
    3: [(3, 0, 0), (2, 1, 0), (1, 2, 0), (0, 3, 0), (2, 0, 1), (1, 1, 1), (0, 2, 1),
        (1, 0, 2), (0, 1, 2), (0, 0, 3)],
}
AX = "xyz"


def carts(n):
    return [(x, y, n - x - y) for x in range(n, -1, -1) for y in range(n - x, -1, -1)]


def nm(t):
    return "%d%d%d" % t


def sub(t, i, k=1):
    l = list(t)
    l[i] -= k
    return tuple(l)


def add(t, i, k=1):
    l = list(t)
    l[i] += k
    return tuple(l)


def classes(lmax):
    """Canonical classes: LA>=LB, LC>=LD, (LA+LB,LA,LB) >= (LC+LD,LC,LD)."""
    pairs = [(a, b) for a in range(lmax + 1) for b in range(a + 1)]
    key = lambda p: (p[0] + p[1], p[0], p[1])
    out = []
    for p in pairs:
        for q in pairs:
            if key(p) >= key(q):
                out.append(p + q)
    return out


def pair_types(lmax):
    return sorted([(a, b) for a in range(lmax + 1) for b in range(a + 1)],
                  key=lambda p: (p[0] + p[1], p[0], p[1]))


class VRR:
    """Dependency-driven emission of [e0|f0]^(m)."""

    def __init__(self, prec="double"):
        self.memo = {}
        self.lines = []
        self.prec = prec
        self.sfx = "f" if prec == "float" else ""
        self.nflops = 0

    def get(self, e, f, m):
        if min(e) < 0 or min(f) < 0:
            return None
        key = (e, f, m)
        if key in self.memo:
            return self.memo[key]
        if sum(e) == 0 and sum(f) == 0:
            name = "F%d" % m
            self.memo[key] = name
            return name
        terms = []
        if sum(f) > 0:
            i = [k for k in range(3) if f[k] > 0][0]
            f1 = sub(f, i)
            a = self.get(e, f1, m)
            b = self.get(e, f1, m + 1)
            terms.append("QC%s*%s" % (AX[i], a))
            terms.append("WQ%s*%s" % (AX[i], b))
            if f1[i] > 0:
                f2 = sub(f, i, 2)
                c = self.get(e, f2, m)
                d = self.get(e, f2, m + 1)
                terms.append("%d.0%s*o2q*(%s - rq*%s)" % (f1[i], self.sfx, c, d) if f1[i] > 1 else "o2q*(%s - rq*%s)" % (c, d))
                self.nflops += 4
            if e[i] > 0:
                g = self.get(sub(e, i), f1, m + 1)
                terms.append("%s*%s" % ("%d.0%s*o2pq" % (e[i], self.sfx) if e[i] > 1 else "o2pq", g))
                self.nflops += 2
            self.nflops += 4
        else:
            i = [k for k in range(3) if e[k] > 0][0]
            e1 = sub(e, i)
            a = self.get(e1, f, m)
            b = self.get(e1, f, m + 1)
            terms.append("PA%s*%s" % (AX[i], a))
            terms.append("WP%s*%s" % (AX[i], b))
            if e1[i] > 0:
                e2 = sub(e, i, 2)
                c = self.get(e2, f, m)
                d = self.get(e2, f, m + 1)
                terms.append("%d.0%s*o2p*(%s - rp*%s)" % (e1[i], self.sfx, c, d) if e1[i] > 1 else "o2p*(%s - rp*%s)" % (c, d))
                self.nflops += 4
            self.nflops += 4
        name = "v%s_%s_%d" % (nm(e), nm(f), m)
        self.lines.append("const %s %s = %s;" % (self.prec, name, " + ".join(terms)))
        self.memo[key] = name
        return name


class HRR:
    """(ab|cd) from contracted (e0|f0) accumulators c_<e>_<f>."""

    def __init__(self, prec="double"):
        self.memo = {}
        self.lines = []
        self.nflops = 0
        self.prec = prec

    def get(self, a, b, c, d):
        key = (a, b, c, d)
        if key in self.memo:
            return self.memo[key]
        if sum(d) > 0:
            i = [k for k in range(3) if d[k] > 0][0]
            x = self.get(a, b, add(c, i), sub(d, i))
            y = self.get(a, b, c, sub(d, i))
            expr = "%s + CD%s*%s" % (x, AX[i], y)
        elif sum(b) > 0:
            i = [k for k in range(3) if b[k] > 0][0]
            x = self.get(add(a, i), sub(b, i), c, d)
            y = self.get(a, sub(b, i), c, d)
            expr = "%s + AB%s*%s" % (x, AX[i], y)
        else:
            name = "c_%s_%s" % (nm(a), nm(c))
            self.memo[key] = name
            return name
        self.nflops += 2
        name = "h%s_%s_%s_%s" % (nm(a), nm(b), nm(c), nm(d))
        self.lines.append("const %s %s = %s;" % (self.prec, name, expr))
        self.memo[key] = name
        return name


# gradient classes with total angular momentum >= this get one kernel per
# derivative centre (two accumulator sets each instead of four)
GRAD_SPLIT_L = int(os.environ.get("QB_GRAD_SPLIT_L", "4"))
# f classes with straight-line kernels: total angular momentum up to
# F_MAX_L for the Fock build and the gradient (the larger ones run the
# generic kernels of eri_generic.cu), FP32 variants up to F32_MAX_L (the
# FP32 lists of the classes between run their FP64 kernels)
F_MAX_L = 8
F32_MAX_L = 6


def grad_group_sizes(la, lb, lc, ld):
    """Lanes per shell quartet compiled for a gradient class: 1, 2 and 4 for
    the classes with total angular momentum <= 2 (qb_autotune_grad picks
    one per class), 1 for the others."""
    return [1, 2, 4] if la + lb + lc + ld <= 2 else [1]


def group_sizes(la, lb, lc, ld):
    """Lanes per shell quartet compiled for a class: the light classes, whose
    cost is the primitive loop, get sub-warp groups up to a whole warp; the
    heavy ones, whose cost is the recurrences, one lane per quartet."""
    L = la + lb + lc + ld
    if L <= 2:
        return [1, 2, 4, 8, 16, 32]
    if L <= 4:
        return [1, 2, 4, 8]
    return [1]


# One lane per quartet walks its primitive quartets ket-outer, bra-inner
# for the classes up to this total angular momentum (gradient: of the
# underlying class): the list is grouped by bra pair, so the inner loop's
# primitive-pair loads are the same address across the warp (one broadcast
# wavefront) where the bra-inner order made each lane load its own ket's
# records once per bra primitive.  The heavier classes, bound by their
# recurrences and register spills, keep bra-outer.
KET_OUTER_MAX_L = 4


SB_FLAG = 256     # kSbFlag of eri_common.cuh
SB_MAX_L = 2      # kSbMaxL of eri_common.cuh


def sb_group_sizes(la, lb, lc, ld):
    """Lanes per quartet of the staged-Boys kernels of a class (FP64, the
    light classes, whose per-primitive Boys reads are their largest load;
    FP32 variants were measured slower than the plain FP32 kernels on every
    light class of (H2O)32/6-31G** and are not built)."""
    return [1, 2, 4] if la + lb + lc + ld <= SB_MAX_L else []


def class_variants(la, lb, lc, ld):
    """Every launch code of a class the autotuner tries: lanes per quartet,
    then SB_FLAG + lanes for the staged-Boys kernels."""
    return group_sizes(la, lb, lc, ld) + [SB_FLAG + g for g in sb_group_sizes(la, lb, lc, ld)]


def gen_class(la, lb, lc, ld, prec="double", list32_launcher=False):
    """One angular class of the Fock build.  prec = "float": the FP32 variant
    of the mixed-precision split (vertical and horizontal recurrences,
    contraction and Boys function in FP32 from FP64 pair data and geometry;
    the digestion into the Fock matrix stays FP64)."""
    L = la + lb + lc + ld
    f32 = prec == "float"
    R = prec
    sfx = "f" if f32 else ""
    tag = "%d%d%d%d" % (la, lb, lc, ld)
    ebra = [e for n in range(la, la + lb + 1) for e in carts(n)]
    fket = [f for n in range(lc, lc + ld + 1) for f in carts(n)]
    vrr = VRR(prec)
    targets = []
    for e in ebra:
        for f in fket:
            targets.append((e, f, vrr.get(e, f, 0)))
    hrr = HRR(prec)
    A, B, Cc, D = QUICK_ORDER[la], QUICK_ORDER[lb], QUICK_ORDER[lc], QUICK_ORDER[ld]
    vals = {}
    for ia, a in enumerate(A):
        for ib, b in enumerate(B):
            for ic, c in enumerate(Cc):
                for id_, d in enumerate(D):
                    vals[(ia, ib, ic, id_)] = hrr.get(a, b, c, d)
    na, nb, nc, nd = len(A), len(B), len(Cc), len(D)
    o = []
    w = o.append
    w("// generated by gen_eri.py: class (%s %s | %s %s)" % tuple("spdf"[x] for x in (la, lb, lc, ld)))
    w('#include "eri_common.cuh"')
    w("namespace qb {")
    ev = "ClassEval32" if f32 else "ClassEval"
    w("template <> struct %s<%d, %d, %d, %d> {" % (ev, la, lb, lc, ld))
    w("template <int G, int SB = 0>   // SB: Boys records staged in shared memory by the kernel")
    w("__device__ __forceinline__ static void run(const QuartetCtx& q, const FockParams& P, int sub)")
    w("{")
    w("    constexpr int L = %d;" % L)
    for e, f, _ in targets:
        w("    %s c_%s_%s = 0.0%s;" % (R, nm(e), nm(f), sfx))
    body = []
    b = body.append
    if f32:
        # one 32-byte record per primitive pair, FP32 Boys records
        b("const PrimRec32 pk = load_prim32(P.prim32, q.ket_off + ik);")
        b("if (!prim_survives(q, pb.cp, pk.cp, P.prim_limit)) continue;")
        b("PrimQuartet32 s;")
        b("float Fm[L + 1];")
        b("prim_quartet32r<L>(pb, pk, q, P.boys32, s, Fm);")
        b("const float PAx = pb.PAx, PAy = pb.PAy, PAz = pb.PAz;")
        b("const float QCx = pk.PAx, QCy = pk.PAy, QCz = pk.PAz;")
        bra_load = ["const PrimRec32 pb = load_prim32(P.prim32, q.bra_off + ib);"]
        bra_decl = ["PrimRec32 pb = {};"]
        bra_fetch = ["pb = load_prim32(P.prim32, q.bra_off + ib);"]
    else:
        # the ket's three vectors are requested together, ahead of the screen
        b("const double4 xk = load_prim_aux(P.prim, q.ket_off + ik);")
        b("const PrimPair pk = load_prim(P, q.ket_off + ik, xk);")
        b("if (!prim_survives(q, xb.z, xk.z, P.prim_limit)) continue;")
        b("PrimQuartet s;")
        b("double Fm[L + 1];")
        b("prim_quartet<L, SB>(pb, pk, P, s, Fm);")
        b("const double PAx = pb.PAx, PAy = pb.PAy, PAz = pb.PAz;")
        b("const double QCx = pk.PAx, QCy = pk.PAy, QCz = pk.PAz;")
        bra_load = ["const double4 xb = load_prim_aux(P.prim, q.bra_off + ib);",
                    "const PrimPair pb = load_prim(P, q.bra_off + ib, xb);"]
        bra_decl = ["double4 xb = make_double4(0.0, 0.0, 0.0, 0.0);", "PrimPair pb = {};"]
        bra_fetch = ["xb = load_prim_aux(P.prim, q.bra_off + ib);", "pb = load_prim(P, q.bra_off + ib, xb);"]
    b("const %s WPx = s.WPx, WPy = s.WPy, WPz = s.WPz, WQx = s.WQx, WQy = s.WQy, WQz = s.WQz;" % R)
    b("const %s o2p = s.o2p, o2q = s.o2q, o2pq = s.o2pq, rp = s.rp, rq = s.rq;" % R)
    b("(void)PAx; (void)PAy; (void)PAz; (void)QCx; (void)QCy; (void)QCz; (void)WPx; (void)WPy; (void)WPz;")
    b("(void)WQx; (void)WQy; (void)WQz; (void)o2p; (void)o2q; (void)o2pq; (void)rp; (void)rq;")
    for m in range(L + 1):
        b("const %s F%d = Fm[%d];" % (R, m, m))
    body += vrr.lines
    for e, f, v in targets:
        b("c_%s_%s += %s;" % (nm(e), nm(f), v))
    # G == 1: one lane walks the bra x ket primitive double loop
    w("    if constexpr (G == 1) {")
    nkl = 1 if f32 else 2          # the ket record loads that open the body
    if L <= KET_OUTER_MAX_L:
        w("    for (int ik = 0; ik < q.nket; ik++) {")
        for ln in body[:nkl]:
            w("        " + ln)
        w("        for (int ib = 0; ib < q.nbra; ib++) {")
        for ln in bra_load + body[nkl:]:
            w("            " + ln)
        w("        }")
        w("    }")
    else:
        w("    for (int ib = 0; ib < q.nbra; ib++) {")
        for ln in bra_load:
            w("        " + ln)
        w("        for (int ik = 0; ik < q.nket; ik++) {")
        for ln in body:
            w("            " + ln)
        w("        }")
        w("    }")
    # G > 1: the G lanes of a group stride over the flattened primitive
    # quartets (ket fastest); a lane keeps its bra record until its bra
    # primitive changes
    w("    } else {")
    w("    const int nk = q.nket;")
    w("    int ib = nk > 0 ? sub / nk : 0, ik = sub - ib * nk, cur = -1;")
    for ln in bra_decl:
        w("    " + ln)
    w("    for (; nk > 0 && ib < q.nbra; step_pq(ib, ik, G, nk)) {")
    w("        if (ib != cur) {")
    for ln in bra_fetch:
        w("            " + ln)
    w("            cur = ib;")
    w("        }")
    w("        {")
    for ln in body:
        w("            " + ln)
    w("        }")
    w("    }")
    for e, f, _ in targets:
        w("    c_%s_%s = group_sum<G>(c_%s_%s);" % (nm(e), nm(f), nm(e), nm(f)))
    w("    }")
    w("    QuartetCtx qa = q;")
    w("    qa.active = q.active && sub == 0;   // the group's first lane digests")
    dg = []
    w_run = w
    w = dg.append
    if f32:
        w("    const float ABx = (float)q.ABx, ABy = (float)q.ABy, ABz = (float)q.ABz, CDx = (float)q.CDx, CDy = (float)q.CDy, CDz = (float)q.CDz;")
    else:
        w("    const double ABx = q.ABx, ABy = q.ABy, ABz = q.ABz, CDx = q.CDx, CDy = q.CDy, CDz = q.CDz;")
    w("    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;")
    for ln in hrr.lines:
        w("    " + ln)
    # ---- digestion
    w("    // Coulomb / exchange digestion (weights and symmetry in digest_*)")
    w("    const double* __restrict__ Dm = P.dense;")
    w("    const int n = P.nbasis;")
    w("    const int a0 = q.bfA, b0 = q.bfB, c0 = q.bfC, d0 = q.bfD;")

    DT = "float" if f32 else "double"

    def dl(x, y):
        if f32:
            return "(float)__ldg(Dm + (size_t)(%s) * n + (%s))" % (x, y)
        return "__ldg(Dm + (size_t)(%s) * n + (%s))" % (x, y)
    # density loads
    for ic in range(nc):
        for id_ in range(nd):
            w("    const %s Dcd_%d_%d = %s;" % (DT, ic, id_, dl("c0+%d" % ic, "d0+%d" % id_)))
    for ia in range(na):
        for ib in range(nb):
            w("    const %s Dab_%d_%d = %s;" % (DT, ia, ib, dl("a0+%d" % ia, "b0+%d" % ib)))
    w("    if (P.hybrid != 0.0) {")
    # exchange needs D_bd, D_bc, D_ad, D_ac
    Kspec = [("ac", "bd", na, nc, nb, nd), ("ad", "bc", na, nd, nb, nc), ("bc", "ad", nb, nc, na, nd), ("bd", "ac", nb, nd, na, nc)]
    idxmap = {"a": "ia", "b": "ib", "c": "ic", "d": "id_"}
    bases = {"a": "a0", "b": "b0", "c": "c0", "d": "d0"}
    sizes = {"a": na, "b": nb, "c": nc, "d": nd}
    # load the four exchange density blocks
    for blk in ("bd", "bc", "ad", "ac"):
        x, y = blk
        for i in range(sizes[x]):
            for j in range(sizes[y]):
                w("        const %s D%s_%d_%d = %s;" % (DT, blk, i, j, dl("%s+%d" % (bases[x], i), "%s+%d" % (bases[y], j))))
    for out_blk, d_blk, n1, n2, m1, m2 in Kspec:
        x, y = out_blk
        u, v = d_blk
        for i in range(n1):
            for j in range(n2):
                terms = []
                for k in range(m1):
                    for l in range(m2):
                        idx = {x: i, y: j, u: k, v: l}
                        key = (idx["a"], idx["b"], idx["c"], idx["d"])
                        terms.append("D%s_%d_%d*%s" % (d_blk, k, l, vals[key]))
                w("        const %s K%s_%d_%d = %s;" % (DT, out_blk, i, j, " + ".join(terms)))
    for out_blk, _, n1, n2, _, _ in Kspec:
        x, y = out_blk
        for i in range(n1):
            for j in range(n2):
                w("        digest_exchange(P, qa, %s+%d, %s+%d, K%s_%d_%d);" % (bases[x], i, bases[y], j, out_blk, i, j))
    w("    }")
    # Coulomb
    for ia in range(na):
        for ib in range(nb):
            terms = ["Dcd_%d_%d*%s" % (ic, id_, vals[(ia, ib, ic, id_)]) for ic in range(nc) for id_ in range(nd)]
            w("    const %s Jab_%d_%d = %s;" % (DT, ia, ib, " + ".join(terms)))
    for ic in range(nc):
        for id_ in range(nd):
            terms = ["Dab_%d_%d*%s" % (ia, ib, vals[(ia, ib, ic, id_)]) for ia in range(na) for ib in range(nb)]
            w("    const %s Jcd_%d_%d = %s;" % (DT, ic, id_, " + ".join(terms)))
    w("    const bool bra_uniform = warp_bra_uniform(qa);")
    for ia in range(na):
        for ib in range(nb):
            w("    digest_coulomb_bra(P, qa, a0+%d, b0+%d, Jab_%d_%d, bra_uniform);" % (ia, ib, ia, ib))
    for ic in range(nc):
        for id_ in range(nd):
            w("    digest_coulomb(P, qa, c0+%d, d0+%d, Jcd_%d_%d);" % (ic, id_, ic, id_))
    w = w_run
    for ln in dg:
        w(ln)
    w("}")
    if not f32:
        # store(): the block's unique integrals for QUICK's stored-integral
        # path (gpu_aoint_), one lane per quartet, instead of the digestion
        w("__device__ __forceinline__ static void store(const QuartetCtx& q, const FockParams& P, const AoIntOut& O)")
        w("{")
        w("    constexpr int L = %d;" % L)
        w("    constexpr int SB = 0;   // the Boys table from global memory")
        for e, f, _ in targets:
            w("    double c_%s_%s = 0.0;" % (nm(e), nm(f)))
        w("    for (int ib = 0; ib < q.nbra; ib++) {")
        for ln in bra_load:
            w("        " + ln)
        w("        for (int ik = 0; ik < q.nket; ik++) {")
        for ln in body:
            w("            " + ln)
        w("        }")
        w("    }")
        w("    if (!q.active) return;")
        w("    const double ABx = q.ABx, ABy = q.ABy, ABz = q.ABz, CDx = q.CDx, CDy = q.CDy, CDz = q.CDz;")
        w("    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;")
        for ln in hrr.lines:
            w("    " + ln)
        w("    const int a0 = q.bfA, b0 = q.bfB, c0 = q.bfC, d0 = q.bfD;")
        for ia in range(na):
            for ib in range(nb):
                for ic in range(nc):
                    for id_ in range(nd):
                        w("    aoint_emit(O, q, a0+%d, b0+%d, c0+%d, d0+%d, %s);" % (ia, ib, ic, id_, vals[(ia, ib, ic, id_)]))
        w("}")
    w("};")
    gs = group_sizes(la, lb, lc, ld)
    kname = "fock_class_kernel32" if f32 else "fock_class_kernel"
    w("// lanes per shell quartet compiled for this class: %s" % ", ".join(str(g) for g in gs))
    w("int launch_%s%s(const FockParams& P, int cls, int G, int nq, int nsm, cudaStream_t st)" % (tag, "_f32" if f32 else ""))
    w("{")
    w("    switch (G) {")
    if not f32:
        w("    case -1: { auto kern = aoint_class_kernel<%d, %d, %d, %d>; QB_LAUNCH(kern, class_grid(nq, 1, nsm), 128, 0, st, P, cls, *g_aoint_out); return -1; }"
          % (la, lb, lc, ld))
    for g in gs:
        w("    case %d: { auto kern = %s<%d, %d, %d, %d, %d>; QB_LAUNCH(kern, class_grid(nq, %d, nsm), 128, 0, st, P, cls%s); return %d; }"
          % (g, kname, la, lb, lc, ld, g, g, "" if f32 else ", 0", g))
    for g in ([] if f32 else sb_group_sizes(la, lb, lc, ld)):
        # staged-Boys variant (eri_common.cuh): code kSbFlag + lanes per quartet
        w("    case %d: { auto kern = fock_class_kernel_sb<%d, %d, %d, %d, %d>; static const bool a_ = "
          "cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kBoysSmemBytes) == cudaSuccess; (void)a_; "
          "QB_LAUNCH(kern, class_grid_sb(nq, %d, nsm, kSbBlock, 2), kSbBlock, kBoysSmemBytes, st, P, cls, 0); return %d; }"
          % (SB_FLAG + g, la, lb, lc, ld, g, g, SB_FLAG + g))
    w("    default: { auto kern = %s<%d, %d, %d, %d, 1>; QB_LAUNCH(kern, class_grid(nq, 1, nsm), 128, 0, st, P, cls%s); return 1; }"
      % (kname, la, lb, lc, ld, "" if f32 else ", 0"))
    w("    }")
    w("}")
    if list32_launcher:
        # no FP32 kernel for this class: its FP32 list runs in FP64
        w("int launch_%s_f32(const FockParams& P, int cls, int G, int nq, int nsm, cudaStream_t st)" % tag)
        w("{")
        w("    (void)G;")
        w("    auto kern = fock_class_kernel<%d, %d, %d, %d, 1>;" % (la, lb, lc, ld))
        w("    QB_LAUNCH(kern, class_grid(nq, 1, nsm), 128, 0, st, P, cls, 1);")
        w("    return 1;")
        w("}")
    w("}  // namespace qb")
    stats = dict(vrr_flops=vrr.nflops, vrr_nodes=len(vrr.lines), hrr_flops=hrr.nflops, targets=len(targets),
                 ncomp=na * nb * nc * nd)
    return "\n".join(o) + "\n", stats


def gen_grad_class(la, lb, lc, ld, part=0, prec="double"):
    """Nuclear gradient of the two-electron energy for one class: derivative
    integrals from exponent-weighted contractions,
      d/dA (ab|cd) = (a+1 b|cd)_{2 alpha} - a_i (a-1 b|cd),
      d/dB (ab|cd) = (a b+1|cd)_{2 beta}  - b_i (a b-1|cd),
      d/dC (ab|cd) = (ab|c+1 d)_{2 gamma} - c_i (ab|c-1 d),   d/dD = -(A+B+C)
    (QUICK: gpu_get2e_subs_grad.h:143-512, storeAA/BB/CC), contracted with
    Gamma = w [4 D_ab D_cd - h (D_ac D_bd + D_ad D_bc)], the sum of the
    energy's density factors over the eight index permutations.
    prec = "float": the FP32 kernel of the mixed split (FP32 primitive and
    Boys records, recurrences, transfer and density products in FP32; the
    twelve numbers of a quartet are added to the gradient in FP64)."""
    L = la + lb + lc + ld + 1
    f32 = prec == "float"
    R = prec
    sfx = "f" if f32 else ""
    tag = "%d%d%d%d" % (la, lb, lc, ld) + ("" if part == 0 else "_" + "abc"[part - 1])
    rng = lambda lo, hi: [e for n in range(max(lo, 0), hi + 1) for e in carts(n)]
    want = {"s0": True, "sa": part in (0, 1), "sb": part in (0, 2), "sc": part in (0, 3)}
    S0e, S0f = rng(la - 1, la + lb), rng(lc - 1, lc + ld)
    SAe, SAf = rng(la + 1, la + lb + 1), rng(lc, lc + ld)
    SBe, SBf = rng(la, la + lb + 1), rng(lc, lc + ld)
    SCe, SCf = rng(la, la + lb), rng(lc + 1, lc + ld + 1)
    vrr = VRR(prec)
    acc = {}
    for nmz, es, fs in (("s0", S0e, S0f), ("sa", SAe, SAf), ("sb", SBe, SBf), ("sc", SCe, SCf)):
        if want[nmz]:
            acc[nmz] = [(e, f, None) for e in es for f in fs]
    hrrs = {k: HRRX(k, prec) for k in acc}
    A, B, Cc, D = QUICK_ORDER[la], QUICK_ORDER[lb], QUICK_ORDER[lc], QUICK_ORDER[ld]
    na, nb, nc, nd = len(A), len(B), len(Cc), len(D)
    deriv = {}
    for ia, a in enumerate(A):
        for ib, b in enumerate(B):
            for ic, c in enumerate(Cc):
                for id_, d in enumerate(D):
                    for i in range(3):
                        ta = tb = tc = ["0.0" + sfx]
                        if want["sa"]:
                            ta = [hrrs["sa"].get(add(a, i), b, c, d)]
                            if a[i] > 0:
                                ta.append("-%d.0%s*%s" % (a[i], sfx, hrrs["s0"].get(sub(a, i), b, c, d)))
                        if want["sb"]:
                            tb = [hrrs["sb"].get(a, add(b, i), c, d)]
                            if b[i] > 0:
                                tb.append("-%d.0%s*%s" % (b[i], sfx, hrrs["s0"].get(a, sub(b, i), c, d)))
                        if want["sc"]:
                            tc = [hrrs["sc"].get(a, b, add(c, i), d)]
                            if c[i] > 0:
                                tc.append("-%d.0%s*%s" % (c[i], sfx, hrrs["s0"].get(a, b, sub(c, i), d)))
                        deriv[(ia, ib, ic, id_, i)] = (" + ".join(ta), " + ".join(tb), " + ".join(tc))
    # only the accumulators the horizontal recurrence reads, and only their
    # vertical-recurrence targets
    used = set()
    for h in hrrs.values():
        used |= set(h.leaves)
    for k in list(acc):
        acc[k] = [(e, f, vrr.get(e, f, 0)) for e, f, _ in acc[k] if "%s_%s_%s" % (k, nm(e), nm(f)) in used]
    o = []
    w = o.append
    w("// generated by gen_eri.py: gradient class (%s %s | %s %s)" % tuple("spdf"[x] for x in (la, lb, lc, ld)))
    w('#include "eri_common.cuh"')
    w('#include "grad_common.cuh"')
    w("namespace qb {")
    w("template <> struct %s<%d, %d, %d, %d, %d> {" % ("GradEval32" if f32 else "GradEval", la, lb, lc, ld, part))
    # the primitive-quartet body of run<GS>
    if f32:
        inner = ["PrimQuartet32 s;", "float Fm[L + 1];", "prim_quartet32r<L>(pb, pk, q, P.boys32, s, Fm);"]
    else:
        inner = ["PrimQuartet s;", "double Fm[L + 1];", "prim_quartet<L>(pb, pk, P, s, Fm);"]
    inner += ["const %s PAx = pb.PAx, PAy = pb.PAy, PAz = pb.PAz;" % R,
             "const %s QCx = pk.PAx, QCy = pk.PAy, QCz = pk.PAz;" % R,
             "const %s WPx = s.WPx, WPy = s.WPy, WPz = s.WPz, WQx = s.WQx, WQy = s.WQy, WQz = s.WQz;" % R,
             "const %s o2p = s.o2p, o2q = s.o2q, o2pq = s.o2pq, rp = s.rp, rq = s.rq;" % R,
             "(void)PAx; (void)PAy; (void)PAz; (void)QCx; (void)QCy; (void)QCz; (void)WPx; (void)WPy; (void)WPz;",
             "(void)WQx; (void)WQy; (void)WQz; (void)o2p; (void)o2q; (void)o2pq; (void)rp; (void)rq;"]
    inner += ["const %s F%d = Fm[%d];" % (R, m, m) for m in range(L + 1)]
    inner += list(vrr.lines)
    wt = {"s0": "", "sa": "a2*", "sb": "b2*", "sc": "c2*"}
    for k, lst in acc.items():
        for e, f, v in lst:
            inner.append("%s_%s_%s += %s%s;" % (k, nm(e), nm(f), wt[k], v))
    # after the contraction: horizontal recurrence, density products, digestion
    tail = []
    t_ = tail.append
    if f32:
        t_("    const float ABx = (float)q.ABx, ABy = (float)q.ABy, ABz = (float)q.ABz, CDx = (float)q.CDx, CDy = (float)q.CDy, CDz = (float)q.CDz;")
    else:
        t_("    const double ABx = q.ABx, ABy = q.ABy, ABz = q.ABz, CDx = q.CDx, CDy = q.CDy, CDz = q.CDz;")
    t_("    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;")
    for h in hrrs.values():
        for ln in h.lines:
            t_("    " + ln)
    t_("    const double* __restrict__ Dm = P.dense;")
    t_("    const int n = P.nbasis;")
    t_("    const int a0 = q.bfA, b0 = q.bfB, c0 = q.bfC, d0 = q.bfD;")
    t_("    const %s hx = (%s)P.hybrid;" % (R, R))

    def dl(x, y):
        if f32:
            return "(float)__ldg(Dm + (size_t)(%s) * n + (%s))" % (x, y)
        return "__ldg(Dm + (size_t)(%s) * n + (%s))" % (x, y)
    bases = {"a": "a0", "b": "b0", "c": "c0", "d": "d0"}
    sizes = {"a": na, "b": nb, "c": nc, "d": nd}
    for blk in ("ab", "cd", "ac", "bd", "ad", "bc"):
        x, y = blk
        for i in range(sizes[x]):
            for j in range(sizes[y]):
                t_("    const %s D%s_%d_%d = %s;" % (R, blk, i, j, dl("%s+%d" % (bases[x], i), "%s+%d" % (bases[y], j))))
    t_("    %s gA[3] = {0.0%s, 0.0%s, 0.0%s}, gB[3] = {0.0%s, 0.0%s, 0.0%s}, gC[3] = {0.0%s, 0.0%s, 0.0%s};" % ((R,) + (sfx,) * 9))
    for ia in range(na):
        for ib in range(nb):
            for ic in range(nc):
                for id_ in range(nd):
                    t_("    {")
                    t_("        const %s g = 4.0%s*Dab_%d_%d*Dcd_%d_%d - hx*(Dac_%d_%d*Dbd_%d_%d + Dad_%d_%d*Dbc_%d_%d);" % (
                        R, sfx, ia, ib, ic, id_, ia, ic, ib, id_, ia, id_, ib, ic))
                    for i in range(3):
                        da, db, dc = deriv[(ia, ib, ic, id_, i)]
                        t_("        gA[%d] += g*(%s); gB[%d] += g*(%s); gC[%d] += g*(%s);" % (i, da, i, db, i, dc))
                    t_("    }")
    w("template <int GS>")
    w("__device__ __forceinline__ static void run(const QuartetCtx& q, const FockParams& P, const GradExtra& G, int sub)")
    w("{")
    w("    constexpr int L = %d;" % L)
    for k, lst in acc.items():
        for e, f, _ in lst:
            w("    %s %s_%s_%s = 0.0%s;" % (R, k, nm(e), nm(f), sfx))
    if f32:
        bra = ["const PrimRec32 pb = load_prim32(P.prim32, q.bra_off + ib);",
               "const float a2 = 2.0f * pb.alpha;",
               "const float b2 = 2.0f * pb.p - a2;"]
        ket = ["const PrimRec32 pk = load_prim32(P.prim32, q.ket_off + ik);",
               "if (!prim_survives(q, pb.cp, pk.cp, P.prim_limit)) continue;",
               "const float c2 = 2.0f * pk.alpha;"]
    else:
        bra = ["const double4 xb = load_prim_aux(P.prim, q.bra_off + ib);",
               "const PrimPair pb = load_prim(P, q.bra_off + ib, xb);",
               "const double a2 = 2.0 * xb.y;",
               "const double b2 = 2.0 * pb.p - a2;"]
        ket = ["const double4 xk = load_prim_aux(P.prim, q.ket_off + ik);",
               "const PrimPair pk = load_prim(P, q.ket_off + ik, xk);",
               "if (!prim_survives(q, xb.z, xk.z, P.prim_limit)) continue;",
               "const double c2 = 2.0 * xk.y;"]
    # one lane per quartet: the bra x ket primitive double loop (each bra
    # record read once); GS lanes: they stride over the flattened primitive
    # quartets
    w("    if constexpr (GS == 1) {")
    if L - 1 <= KET_OUTER_MAX_L:
        # ket-outer (KET_OUTER_MAX_L): the screen needs both records, so it
        # moves into the inner loop
        kload = [ln for ln in ket if "prim_survives" not in ln]
        screen = [ln for ln in ket if "prim_survives" in ln]
        w("    for (int ik = 0; ik < q.nket; ik++) {")
        for ln in kload:
            w("        " + ln)
        w("        for (int ib = 0; ib < q.nbra; ib++) {")
        for ln in bra + screen + inner:
            w("            " + ln)
        w("        }")
        w("    }")
    else:
        w("    for (int ib = 0; ib < q.nbra; ib++) {")
        for ln in bra:
            w("        " + ln)
        w("        for (int ik = 0; ik < q.nket; ik++) {")
        for ln in ket + inner:
            w("            " + ln)
        w("        }")
        w("    }")
    w("    } else {")
    w("    const int nk = q.nket, npq = q.nbra * nk;")
    w("    for (int t = sub; t < npq; t += GS) {")
    w("        const int ib = t / nk, ik = t - ib * nk;")
    for ln in bra:
        w("        " + ln)
    w("        {")
    for ln in ket + inner:
        w("            " + ln)
    w("        }")
    w("    }")
    w("    }")
    w("    if constexpr (GS > 1) {")
    for k, lst in acc.items():
        for e, f, _ in lst:
            w("        %s_%s_%s = group_sum<GS>(%s_%s_%s);" % (k, nm(e), nm(f), k, nm(e), nm(f)))
    w("    }")
    w("    QuartetCtx qa = q;")
    w("    qa.active = q.active && sub == 0;   // the group's first lane digests")
    for ln in tail:
        w(ln)
    if f32:
        w("    const double dA[3] = {gA[0], gA[1], gA[2]}, dB[3] = {gB[0], gB[1], gB[2]}, dC[3] = {gC[0], gC[1], gC[2]};")
        w("    grad_digest<%d>(qa, G, dA, dB, dC);" % part)
    else:
        w("    grad_digest<%d>(qa, G, gA, gB, gC);" % part)
    w("}")
    w("};")
    gs = grad_group_sizes(la, lb, lc, ld)
    w("// lanes per shell quartet compiled for this class: %s" % ", ".join(str(x) for x in gs))
    kname = "grad_class_kernel32" if f32 else "grad_class_kernel"
    w("int launch_grad%s_%s(const FockParams& P, const GradExtra& G, int cls, int GS, int nq, int nsm, cudaStream_t st)" % ("32" if f32 else "", tag))
    w("{")
    w("    switch (GS) {")
    for x in gs:
        w("    case %d: { auto kern = %s<%d, %d, %d, %d, %d, %d>; QB_LAUNCH(kern, class_grid(nq, %d, nsm), 128, grad_smem(G), st, P, G, cls); return %d; }"
          % (x, kname, la, lb, lc, ld, part, x, x, x))
    w("    default: { auto kern = %s<%d, %d, %d, %d, %d, 1>; QB_LAUNCH(kern, class_grid(nq, 1, nsm), 128, grad_smem(G), st, P, G, cls); return 1; }"
      % (kname, la, lb, lc, ld, part))
    w("    }")
    w("}")
    w("}  // namespace qb")
    return "\n".join(o) + "\n", dict(vrr_flops=vrr.nflops, hrr_flops=sum(h.nflops for h in hrrs.values()),
                                      lines=len(o))


class HRRX(HRR):
    """HRR over one named accumulator set (prefix_<e>_<f> leaves)."""

    def __init__(self, prefix, prec="double"):
        HRR.__init__(self, prec)
        self.prefix = prefix
        self.leaves = set()

    def get(self, a, b, c, d):
        key = (a, b, c, d)
        if key in self.memo:
            return self.memo[key]
        if sum(d) > 0:
            i = [k for k in range(3) if d[k] > 0][0]
            x = self.get(a, b, add(c, i), sub(d, i))
            y = self.get(a, b, c, sub(d, i))
            expr = "%s + CD%s*%s" % (x, AX[i], y)
        elif sum(b) > 0:
            i = [k for k in range(3) if b[k] > 0][0]
            x = self.get(add(a, i), sub(b, i), c, d)
            y = self.get(a, sub(b, i), c, d)
            expr = "%s + AB%s*%s" % (x, AX[i], y)
        else:
            name = "%s_%s_%s" % (self.prefix, nm(a), nm(c))
            self.leaves.add(name)
            self.memo[key] = name
            return name
        self.nflops += 2
        name = "%s_h%s_%s_%s_%s" % (self.prefix, nm(a), nm(b), nm(c), nm(d))
        self.lines.append("const %s %s = %s;" % (self.prec, name, expr))
        self.memo[key] = name
        return name


def gen_schwarz(la, lb):
    """Diagonal (ab|ab) blocks for QUICK's Schwarz bounds (schwarz.f90:46-548):
    max over components of |(ab|ab)| cons(a)^2 cons(b)^2, either contracted
    (mode 0, one thread per shell pair) or for a single primitive pair on both
    sides (mode 1, one thread per primitive pair)."""
    L = 2 * (la + lb)
    tag = "%d%d" % (la, lb)
    ebra = [e for n in range(la, la + lb + 1) for e in carts(n)]
    vrr = VRR()
    targets = []
    for e in ebra:
        for f in ebra:
            targets.append((e, f, vrr.get(e, f, 0)))
    hrr = HRR()
    A, B = QUICK_ORDER[la], QUICK_ORDER[lb]
    diag = []
    for ia, a in enumerate(A):
        for ib, b in enumerate(B):
            diag.append((ia, ib, hrr.get(a, b, a, b)))
    o = []
    w = o.append
    w("// generated by gen_eri.py: Schwarz diagonal (%s %s | %s %s)" % tuple("spdf"[x] for x in (la, lb, la, lb)))
    w('#include "eri_common.cuh"')
    w('#include "schwarz.cuh"')
    w("namespace qb {")
    w("template <> __device__ __forceinline__ double schwarz_diag<%d, %d>(const SchwarzParams& S, int rec, int p0, int np)" % (la, lb))
    w("{")
    w("    constexpr int L = %d;" % L)
    w("    const int4 info = S.pair_bf[rec];")
    w("    const double4 ab = S.pair_AB[rec];")
    w("    FockParams P;")
    w("    P.boys = S.boys;")
    for e, f, _ in targets:
        w("    double c_%s_%s = 0.0;" % (nm(e), nm(f)))
    w("    for (int ib = p0; ib < p0 + np; ib++) {")
    w("        const PrimPair pb = load_prim_tab(S.prim, info.z + ib, load_prim_aux(S.prim, info.z + ib));")
    w("        for (int ik = p0; ik < p0 + np; ik++) {")
    w("            const PrimPair pk = load_prim_tab(S.prim, info.z + ik, load_prim_aux(S.prim, info.z + ik));")
    w("            PrimQuartet s;")
    w("            double Fm[L + 1];")
    w("            prim_quartet<L>(pb, pk, P, s, Fm);")
    w("            const double PAx = pb.PAx, PAy = pb.PAy, PAz = pb.PAz;")
    w("            const double QCx = pk.PAx, QCy = pk.PAy, QCz = pk.PAz;")
    w("            const double WPx = s.WPx, WPy = s.WPy, WPz = s.WPz, WQx = s.WQx, WQy = s.WQy, WQz = s.WQz;")
    w("            const double o2p = s.o2p, o2q = s.o2q, o2pq = s.o2pq, rp = s.rp, rq = s.rq;")
    w("            (void)PAx; (void)PAy; (void)PAz; (void)QCx; (void)QCy; (void)QCz; (void)WPx; (void)WPy; (void)WPz;")
    w("            (void)WQx; (void)WQy; (void)WQz; (void)o2p; (void)o2q; (void)o2pq; (void)rp; (void)rq;")
    for m in range(L + 1):
        w("            const double F%d = Fm[%d];" % (m, m))
    for ln in vrr.lines:
        w("            " + ln)
    for e, f, v in targets:
        w("            c_%s_%s += %s;" % (nm(e), nm(f), v))
    w("        }")
    w("    }")
    w("    const double ABx = ab.x, ABy = ab.y, ABz = ab.z, CDx = ab.x, CDy = ab.y, CDz = ab.z;")
    w("    (void)ABx; (void)ABy; (void)ABz; (void)CDx; (void)CDy; (void)CDz;")
    for ln in hrr.lines:
        w("    " + ln)
    w("    double m = 0.0;")
    for ia, ib, v in diag:
        w("    { const double ca = S.cons[info.x + %d], cb = S.cons[info.y + %d]; m = fmax(m, fabs(%s) * ca * ca * cb * cb); }" % (ia, ib, v))
    w("    return m;")
    w("}")
    w("void launch_schwarz_%s(const SchwarzParams& S, int begin, int end, int mode, int grid, int block, cudaStream_t st)" % tag)
    w("{")
    w("    auto kern = schwarz_kernel<%d, %d>;" % (la, lb))
    w("    QB_LAUNCH(kern, grid, block, 0, st, S, begin, end, mode);")
    w("}")
    w("}  // namespace qb")
    return "\n".join(o) + "\n"


def write_if_changed(path, src):
    old = open(path).read() if os.path.exists(path) else None
    if old != src:
        with open(path, "w") as fh:
            fh.write(src)


def class_stats(la, lb, lc, ld):
    """FLOP counts of a class without emitting code (for the classes the
    generic kernel runs)."""
    vrr = VRR()
    for n1 in range(la, la + lb + 1):
        for e in carts(n1):
            for n2 in range(lc, lc + ld + 1):
                for f in carts(n2):
                    vrr.get(e, f, 0)
    hrr = HRR()
    A, B, Cc, D = QUICK_ORDER[la], QUICK_ORDER[lb], QUICK_ORDER[lc], QUICK_ORDER[ld]
    for a in A:
        for b in B:
            for c in Cc:
                for d in D:
                    hrr.get(a, b, c, d)
    ntar = sum(len(carts(n)) for n in range(la, la + lb + 1)) * sum(len(carts(n)) for n in range(lc, lc + ld + 1))
    return dict(vrr_flops=vrr.nflops, vrr_nodes=len(vrr.lines), hrr_flops=hrr.nflops, targets=ntar,
                ncomp=len(A) * len(B) * len(Cc) * len(D))


def main(outdir, lmax=2, lmax_all=3):
    """Straight-line kernels for the classes with every shell <= lmax; the
    class table covers shells up to lmax_all (the rest run the generic
    kernel, eri_generic.cu)."""
    os.makedirs(outdir, exist_ok=True)
    cls_all = classes(lmax_all)
    # straight-line kernels: every class up to lmax, and the f classes whose
    # total angular momentum is at most F_MAX_L (the larger ones run the
    # generic kernel; their straight-line code spills most of its values)
    cls = [c for c in cls_all if max(c) <= lmax or sum(c) <= F_MAX_L]
    cls32 = set(c for c in cls if max(c) <= lmax or sum(c) <= F32_MAX_L)
    # gradient: the same classes (the larger ones run the generic gradient
    # kernel, eri_generic.cu, which is slow for the many small quartets)
    cls_grad = list(cls)
    lines = ["// generated by gen_eri.py", "#pragma once", "namespace qb {",
             "static const int kNumClasses = %d;" % len(cls_all),
             "static const int kClassL[%d][4] = {%s};" % (len(cls_all), ", ".join("{%d,%d,%d,%d}" % c for c in cls_all)),
             "static const int kNumPairTypes = %d;" % len(pair_types(lmax_all)),
             "static const int kPairTypeL[%d][2] = {%s};" % (len(pair_types(lmax_all)), ", ".join("{%d,%d}" % p for p in pair_types(lmax_all))),
             "static const int kGeneratedLmax = %d;   // classes above run the generic kernel" % lmax,
             "// 1: the class has no straight-line kernel and runs the generic one (eri_generic.cu)",
             "static const int kClassGeneric[%d] = {%s};" % (
                 len(cls_all), ", ".join("0" if c in set(cls) else "1" for c in cls_all)),
             "}"]
    with open(os.path.join(outdir, "eri_classes.h"), "w") as fh:
        fh.write("\n".join(lines) + "\n")
    stats = {}
    for c in cls:
        src, st = gen_class(*c, list32_launcher=c not in cls32)
        stats[c] = st
        write_if_changed(os.path.join(outdir, "eri_%d%d%d%d.cu" % c), src)
        if c in cls32:
            src32, _ = gen_class(*c, prec="float")
            write_if_changed(os.path.join(outdir, "eri32_%d%d%d%d.cu" % c), src32)
        elif os.path.exists(os.path.join(outdir, "eri32_%d%d%d%d.cu" % c)):
            os.remove(os.path.join(outdir, "eri32_%d%d%d%d.cu" % c))
    # launch table
    lt = ['#include "eri_common.cuh"', '#include "eri_classes.h"', "namespace qb {"]
    for c in cls:
        lt.append("int launch_%d%d%d%d(const FockParams& P, int cls, int G, int nq, int nsm, cudaStream_t st);" % c)
        lt.append("int launch_%d%d%d%d_f32(const FockParams& P, int cls, int G, int nq, int nsm, cudaStream_t st);" % c)
    lt.append("int launch_generic_class(int cls, int la, int lb, int lc, int ld, const FockParams& P, int nq, int nsm, "
              "int fp32_list, cudaStream_t st);")
    gen_set = set(cls)
    lt += ["int launch_class(int cls, const FockParams& P, int G, int nq, int nsm, cudaStream_t st)", "{",
           "    switch (cls) {"]
    for k, c in enumerate(cls_all):
        if c in gen_set:
            lt.append("    case %d: return launch_%d%d%d%d(P, %d, G, nq, nsm, st);" % ((k,) + c + (k,)))
        else:
            lt.append("    case %d: return launch_generic_class(%d, %d, %d, %d, %d, P, nq, nsm, 0, st);" % ((k, k) + c))
    lt += ["    default: return 0;", "    }", "}"]
    lt += ["int launch_class32(int cls, const FockParams& P, int G, int nq, int nsm, cudaStream_t st)", "{",
           "    switch (cls) {"]
    for k, c in enumerate(cls_all):
        if c in gen_set:
            lt.append("    case %d: return launch_%d%d%d%d_f32(P, %d, G, nq, nsm, st);" % ((k,) + c + (k,)))
        else:
            lt.append("    case %d: return launch_generic_class(%d, %d, %d, %d, %d, P, nq, nsm, 1, st);" % ((k, k) + c))
    lt += ["    default: return 0;", "    }", "}"]
    lt += ["int class_max_group(int cls)", "{", "    switch (cls) {"]
    for k, c in enumerate(cls_all):
        lt.append("    case %d: return %d;" % (k, max(group_sizes(*c)) if c in gen_set else 1))
    lt += ["    default: return 1;", "    }", "}"]
    lt += ["// launch codes of a class for the autotuner (lanes per quartet, kSbFlag + lanes",
           "// for the staged-Boys kernels); fp32: the FP32 kernels' codes",
           "int class_variants(int cls, int fp32, int* codes, int cap)", "{", "    int n = 0;", "    switch (cls) {"]
    for k, c in enumerate(cls_all):
        if c not in gen_set:
            continue
        v64 = class_variants(*c)
        v32 = group_sizes(*c) if c in cls32 else [1]
        lt.append("    case %d: { static const int a[] = {%s}, b[] = {%s}; const int* v = fp32 ? b : a; n = fp32 ? %d : %d; "
                  "for (int i = 0; i < n && i < cap; i++) codes[i] = v[i]; break; }"
                  % (k, ", ".join(map(str, v64)), ", ".join(map(str, v32)), len(v32), len(v64)))
    lt += ["    default: if (cap > 0) codes[0] = 1; n = 1; break;", "    }", "    return n < cap ? n : cap;", "}",
           "}  // namespace qb"]
    write_if_changed(os.path.join(outdir, "eri_launch.cu"), "\n".join(lt) + "\n")
    import json
    for c in cls_all:
        if c not in stats:
            stats[c] = class_stats(*c)
    write_if_changed(os.path.join(outdir, "class_flops.json"),
                     json.dumps({"%d%d%d%d" % c: s for c, s in stats.items()}, indent=1))
    # gradient kernels, one per class
    gl = ['#include "eri_common.cuh"', '#include "grad_common.cuh"', '#include "eri_classes.h"', "namespace qb {"]
    gstats = {}
    parts = {}
    for c in cls_grad:
        # classes with total angular momentum >= GRAD_SPLIT_L get one kernel
        # per derivative centre (A, B, C): a third of the code and half the
        # accumulators each, which keeps the compile time of the largest
        # classes in minutes and their register spills down
        parts[c] = [0] if sum(c) < GRAD_SPLIT_L else [1, 2, 3]
        for pt in parts[c]:
            src, st_ = gen_grad_class(*c, part=pt)
            tg = "%d%d%d%d" % c + ("" if pt == 0 else "_" + "abc"[pt - 1])
            gstats[tg] = st_
            write_if_changed(os.path.join(outdir, "grad_%s.cu" % tg), src)
            gl.append("int launch_grad_%s(const FockParams& P, const GradExtra& G, int cls, int GS, int nq, int nsm, cudaStream_t st);" % tg)
            if c in cls32:
                src32, _ = gen_grad_class(*c, part=pt, prec="float")
                write_if_changed(os.path.join(outdir, "grad32_%s.cu" % tg), src32)
                gl.append("int launch_grad32_%s(const FockParams& P, const GradExtra& G, int cls, int GS, int nq, int nsm, cudaStream_t st);" % tg)
    gl += ["// returns 0, or -1 for a class without a gradient kernel (f shells)",
           "int launch_grad_class(int cls, const FockParams& P, const GradExtra& G, int GS, int nq, int nsm, cudaStream_t st)",
           "{", "    switch (cls) {"]
    for k, c in enumerate(cls_all):
        if c not in parts:
            continue
        calls = " ".join("launch_grad_%s(P, G, %d, GS, nq, nsm, st);" % ("%d%d%d%d" % c + ("" if pt == 0 else "_" + "abc"[pt - 1]), k)
                         for pt in parts[c])
        gl.append("    case %d: %s return 0;" % (k, calls))
    gl += ["    default: return -1;", "    }", "}"]
    gl += ["// the FP32 kernels of the mixed split, on the class's FP32 list; -1 as above",
           "int launch_grad_class32(int cls, const FockParams& P, const GradExtra& G, int GS, int nq, int nsm, cudaStream_t st)",
           "{", "    switch (cls) {"]
    for k, c in enumerate(cls_all):
        if c not in parts:
            continue
        if c in cls32:
            calls = " ".join("launch_grad32_%s(P, G, %d, GS, nq, nsm, st);" % ("%d%d%d%d" % c + ("" if pt == 0 else "_" + "abc"[pt - 1]), k)
                             for pt in parts[c])
        else:   # no FP32 kernel: the FP64 one on the FP32 list
            calls = "{ GradExtra G32 = G; G32.list32 = 1; %s }" % " ".join(
                "launch_grad_%s(P, G32, %d, GS, nq, nsm, st);" % ("%d%d%d%d" % c + ("" if pt == 0 else "_" + "abc"[pt - 1]), k)
                for pt in parts[c])
        gl.append("    case %d: %s return 0;" % (k, calls))
    gl += ["    default: return -1;", "    }", "}"]
    gl += ["int grad_max_group(int cls)", "{", "    switch (cls) {"]
    for k, c in enumerate(cls_all):
        if c in parts:
            gl.append("    case %d: return %d;" % (k, max(grad_group_sizes(*c))))
    gl += ["    default: return 1;", "    }", "}", "}  // namespace qb"]
    write_if_changed(os.path.join(outdir, "grad_launch.cu"), "\n".join(gl) + "\n")
    write_if_changed(os.path.join(outdir, "grad_flops.json"), json.dumps(gstats, indent=1))
    # per-centre files left over from a build with another split threshold,
    # and FP32 files of classes that have no FP32 kernel now
    for f in os.listdir(outdir):
        for pre in ("grad_", "grad32_"):
            if f.startswith(pre) and f.endswith(".cu") and f != "grad_launch.cu":
                tg = f[len(pre):-3]
                if tg not in gstats or (pre == "grad32_" and tuple(int(ch) for ch in tg[:4]) not in cls32):
                    os.remove(os.path.join(outdir, f))
    # Schwarz kernels, one per pair type
    st = ['#include "eri_common.cuh"', '#include "schwarz.cuh"', '#include "eri_classes.h"', "namespace qb {"]
    for t in pair_types(lmax):
        write_if_changed(os.path.join(outdir, "sch_%d%d.cu" % t), gen_schwarz(*t))
        st.append("void launch_schwarz_%d%d(const SchwarzParams& S, int begin, int end, int mode, int grid, int block, cudaStream_t st);" % t)
    st += ["// returns 0, or -1 for a pair type without a Schwarz kernel (f shells)",
           "int launch_schwarz(int type, const SchwarzParams& S, int begin, int end, int mode, int grid, int block, cudaStream_t st)",
           "{", "    switch (type) {"]
    gen_types = set(pair_types(lmax))
    for k, t in enumerate(pair_types(lmax_all)):
        if t in gen_types:
            st.append("    case %d: launch_schwarz_%d%d(S, begin, end, mode, grid, block, st); return 0;" % ((k,) + t))
    st += ["    default: return -1;", "    }", "}", "}  // namespace qb"]
    write_if_changed(os.path.join(outdir, "sch_launch.cu"), "\n".join(st) + "\n")
    return stats


if __name__ == "__main__":
    lmax = 2
    args = [a for a in sys.argv[1:]]
    if "--lmax" in args:
        k = args.index("--lmax")
        lmax = int(args[k + 1])
        del args[k:k + 2]
    st = main(args[0] if args else "gen", lmax)
    for c, s in st.items():
        print(c, s)
