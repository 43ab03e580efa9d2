// Angular classes with an f shell (any shell up to L = 3): one thread block
// per shell quartet, the recurrences in shared memory.
//
// The straight-line generated kernels (gen_eri.py) cover s, p and d; their
// f counterparts would be tens of thousands of statements per class.  This
// kernel runs the same algorithm with loops instead:
//
//  * F_m(T), m = 0..LA+LB+LC+LD (thread 0, the table scheme of boys<L>);
//  * the Obara-Saika vertical recurrence [e0|f0]^(m), |e| <= LA+LB,
//    |f| <= LC+LD, one level of |f| at a time (three levels kept), the threads
//    of the block sharing each level's entries; a per-class program built
//    once on the host lists every entry with its source offsets in shared
//    memory, so the device loop is loads and FMAs;
//  * contraction of [e0|f0]^(0) for LA <= |e|, LC <= |f| over the primitive
//    quartets that pass QUICK's primitive screen;
//  * the horizontal recurrence in closed form,
//    (a b| = sum_k prod_i C(b_i, k_i) AB_i^(b_i - k_i) (a + k, 0|, first on the
//    ket side for all e, then on the bra side per integral (term lists from
//    the same program);
//  * the quartet's integrals stored in shared memory, then contracted with
//    the density into the six Coulomb/exchange blocks with one thread per
//    output element (no atomics), flushed to the Fock matrix once per quartet
//    with the weights of the generated kernels (digest_coulomb /
//    digest_exchange).
//
// QUICK's own spdf path (gpu_get2e_subs.h:413-850 with int.h's
// vertical_spdf* and the 84 x 84 `store`) computes the same integrals.
#include <algorithm>
#include <cstdlib>
#include <map>
#include <vector>

#include "eri_common.cuh"
#include "grad_common.cuh"
#include "qb_internal.h"
#include "schwarz.cuh"

namespace qb {

constexpr int kGenMaxL = 3;

__host__ __device__ constexpr int g_ncart(int l) { return l < 0 ? 0 : (l + 1) * (l + 2) / 2; }
// number of Cartesians of all levels <= l
__host__ __device__ constexpr int g_ncum(int l) { return l < 0 ? 0 : (l + 1) * (l + 2) * (l + 3) / 6; }

// ------------------------------------------------------------ host side
static int h_lidx(int x, int y, int z)
{
    const int t = y + z;
    (void)x;
    return t * (t + 1) / 2 + z;
}
static void h_cart(int l, int idx, int& x, int& y, int& z)
{
    int t = 0;
    while ((t + 1) * (t + 2) / 2 <= idx) t++;
    z = idx - t * (t + 1) / 2;
    x = l - t;
    y = t - z;
}
static const int kQuickCartH[4][10][3] = {
    {{0, 0, 0}},
    {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}},
    {{2, 0, 0}, {1, 1, 0}, {0, 2, 0}, {1, 0, 1}, {0, 1, 1}, {0, 0, 2}},
    {{3, 0, 0}, {2, 1, 0}, {1, 2, 0}, {0, 3, 0}, {2, 0, 1}, {1, 1, 1}, {0, 2, 1}, {1, 0, 2}, {0, 1, 2}, {0, 0, 3}},
};

// Shared-memory layout of one class (doubles).
struct GenLayout {
    int la, lb, lc, ld;
    int lab, lcd, lt;
    int lvl_off[3];       // three rotating VRR level buffers (level 0 starts with F_m)
    int acc_off, ne, nf;  // contracted [e0|f0], |e| in [la, lab], |f| in [lc, lcd]
    int x_off;            // ket-transformed block X[e][cd] (reuses the level buffers)
    int i_off;            // the quartet's integrals I[ab][cd] (after X, same region)
    int pw_off;           // AB and CD powers, 24 values
    int d_off;            // six density blocks
    int j_off;            // six accumulator blocks
    int total;
};

// The per-class program: every recurrence entry with its source offsets.
struct GenProgram {
    const int* stage;     // nstage x 3: type (0 bra level, 1 ket level, 2 contraction), first entry, count
    int nstage;
    const int4* ent;      // (out, a, c, g) shared-memory offsets; contraction: (acc index, source, -, -)
    const int* meta;      // direction | mul_c << 2 | mul_g << 6 | nm << 10
    const int* kstart;    // ket horizontal terms of component pair cd: [kstart[cd], kstart[cd+1])
    const int4* kterm;    // (f local index, powers of C-D packed 4 bits each, binomial product, -)
    const int* bstart;    // bra horizontal terms of component pair ab
    const int4* bterm;    // (e local index, powers of A-B, binomial product, -)
};

static int level_per_f(int lab, int lt, int k)
{
    int per_f = 0;
    for (int l = 0; l <= lab; l++) per_f += g_ncart(l) * std::max(0, lt - l - k + 1);
    return per_f;
}
static int h_eoff(int lt, int k, int l, int idx)
{
    int off = 0;
    for (int j = 0; j < l; j++) off += g_ncart(j) * (lt - j - k + 1);
    return off + idx * (lt - l - k + 1);
}

static GenLayout gen_layout(int la, int lb, int lc, int ld)
{
    GenLayout G{};
    G.la = la; G.lb = lb; G.lc = lc; G.ld = ld;
    G.lab = la + lb;
    G.lcd = lc + ld;
    G.lt = G.lab + G.lcd;
    int mx = 0;
    for (int k = 0; k <= G.lcd; k++) mx = std::max(mx, level_per_f(G.lab, G.lt, k) * g_ncart(k));
    G.ne = g_ncum(G.lab) - g_ncum(la - 1);
    G.nf = g_ncum(G.lcd) - g_ncum(lc - 1);
    const int nc = g_ncart(lc), nd = g_ncart(ld);
    const int nab = g_ncart(la) * g_ncart(lb);
    const int region = std::max(3 * mx, (G.ne + nab) * nc * nd);
    int off = 0;
    G.lvl_off[0] = 0;
    G.lvl_off[1] = mx;
    G.lvl_off[2] = 2 * mx;
    G.x_off = 0;
    G.i_off = G.ne * nc * nd;
    off = region;
    G.acc_off = off;
    off += G.ne * G.nf;
    G.pw_off = off;
    off += 24;
    const int na = g_ncart(la), nb = g_ncart(lb);
    const int blocks = na * nb + nc * nd + na * nc + na * nd + nb * nc + nb * nd;
    G.d_off = off;
    off += blocks;
    G.j_off = off;
    off += blocks;
    G.total = off;
    return G;
}

struct GenProgramHost {
    std::vector<int> stage, meta, kstart, bstart;
    std::vector<int4> ent, kterm, bterm;
};

static void gen_program(const GenLayout& G, GenProgramHost& H, bool with_hrr = true)
{
    const int lt = G.lt, lab = G.lab;
    auto buf = [&](int k) { return G.lvl_off[k % 3]; };
    auto meta = [](int i, int mc, int mg, int nm) { return i | (mc << 2) | (mg << 6) | (nm << 10); };
    auto push_stage = [&](int type, int start) { H.stage.push_back(type); H.stage.push_back(start);
                                                 H.stage.push_back((int)H.ent.size() - start); };
    // contraction of level k into acc
    auto contract = [&](int k) {
        const int start = (int)H.ent.size();
        const int per_f = level_per_f(lab, lt, k);
        for (int eg = g_ncum(G.la - 1); eg < g_ncum(lab); eg++) {
            int l = 0;
            while (g_ncum(l) <= eg) l++;
            const int eidx = eg - g_ncum(l - 1);
            for (int fidx = 0; fidx < g_ncart(k); fidx++) {
                const int ei = eg - g_ncum(G.la - 1);
                const int fl = g_ncum(k - 1) - g_ncum(G.lc - 1) + fidx;
                const int src = buf(k) + fidx * per_f + h_eoff(lt, k, l, eidx);
                H.ent.push_back(make_int4(ei * G.nf + fl, src, 0, 0));
                H.meta.push_back(0);
            }
        }
        push_stage(2, start);
    };
    // bra levels of level 0: [e0|00]^(m)
    for (int l = 1; l <= lab; l++) {
        const int start = (int)H.ent.size();
        for (int idx = 0; idx < g_ncart(l); idx++) {
            int e[3];
            h_cart(l, idx, e[0], e[1], e[2]);
            const int i = e[0] ? 0 : (e[1] ? 1 : 2);
            int e1[3] = {e[0], e[1], e[2]};
            e1[i]--;
            const int a = buf(0) + h_eoff(lt, 0, l - 1, h_lidx(e1[0], e1[1], e1[2]));
            int c = -1;
            if (e1[i] > 0) {
                int e2[3] = {e1[0], e1[1], e1[2]};
                e2[i]--;
                c = buf(0) + h_eoff(lt, 0, l - 2, h_lidx(e2[0], e2[1], e2[2]));
            }
            H.ent.push_back(make_int4(buf(0) + h_eoff(lt, 0, l, idx), a, c, -1));
            H.meta.push_back(meta(i, e1[i], 0, lt - l + 1));
        }
        push_stage(0, start);
    }
    if (G.lc == 0) contract(0);
    // ket levels
    for (int k = 1; k <= G.lcd; k++) {
        const int start = (int)H.ent.size();
        const int pf0 = level_per_f(lab, lt, k), pf1 = level_per_f(lab, lt, k - 1);
        const int pf2 = k >= 2 ? level_per_f(lab, lt, k - 2) : 0;
        for (int fidx = 0; fidx < g_ncart(k); fidx++) {
            int f[3];
            h_cart(k, fidx, f[0], f[1], f[2]);
            const int i = f[0] ? 0 : (f[1] ? 1 : 2);
            int f1[3] = {f[0], f[1], f[2]};
            f1[i]--;
            const int f1idx = h_lidx(f1[0], f1[1], f1[2]);
            for (int l = 0; l <= lab; l++)
                for (int eidx = 0; eidx < g_ncart(l); eidx++) {
                    int e[3];
                    h_cart(l, eidx, e[0], e[1], e[2]);
                    const int a = buf(k - 1) + f1idx * pf1 + h_eoff(lt, k - 1, l, eidx);
                    int c = -1, g = -1;
                    if (f1[i] > 0) {
                        int f2[3] = {f1[0], f1[1], f1[2]};
                        f2[i]--;
                        c = buf(k - 2) + h_lidx(f2[0], f2[1], f2[2]) * pf2 + h_eoff(lt, k - 2, l, eidx);
                    }
                    if (e[i] > 0) {
                        int e1[3] = {e[0], e[1], e[2]};
                        e1[i]--;
                        g = buf(k - 1) + f1idx * pf1 + h_eoff(lt, k - 1, l - 1, h_lidx(e1[0], e1[1], e1[2]));
                    }
                    H.ent.push_back(make_int4(buf(k) + fidx * pf0 + h_eoff(lt, k, l, eidx), a, c, g));
                    H.meta.push_back(meta(i, f1[i], e[i], lt - l - k + 1));
                }
        }
        push_stage(1, start);
        if (k >= G.lc) contract(k);
    }
    // horizontal terms, closed binomial form
    auto binom = [](int n, int k) { int r = 1; for (int j = 1; j <= k; j++) r = r * (n - k + j) / j; return r; };
    auto terms = [&](int l1, int l2, std::vector<int>& start, std::vector<int4>& out) {
        for (int i1 = 0; i1 < g_ncart(l1); i1++)
            for (int i2 = 0; i2 < g_ncart(l2); i2++) {
                start.push_back((int)out.size());
                const int* A = kQuickCartH[l1][i1];
                const int* B = kQuickCartH[l2][i2];
                for (int kx = 0; kx <= B[0]; kx++)
                    for (int ky = 0; ky <= B[1]; ky++)
                        for (int kz = 0; kz <= B[2]; kz++) {
                            const int x = A[0] + kx, y = A[1] + ky, z = A[2] + kz;
                            const int loc = g_ncum(x + y + z - 1) + h_lidx(x, y, z) - g_ncum(l1 - 1);
                            const int pw = (B[0] - kx) | ((B[1] - ky) << 4) | ((B[2] - kz) << 8);
                            out.push_back(make_int4(loc, pw, binom(B[0], kx) * binom(B[1], ky) * binom(B[2], kz), 0));
                        }
            }
        start.push_back((int)out.size());
    };
    if (!with_hrr) return;   // the gradient program (its shells may exceed f) does its own transfer
    terms(G.lc, G.ld, H.kstart, H.kterm);
    terms(G.la, G.lb, H.bstart, H.bterm);
}

// ------------------------------------------------------------ device side
// F_m(T) times pref for m = 0..L with a runtime L (the scheme of boys<L>).
__device__ void boys_rt(const double* __restrict__ tab, double T, double pref, double* F, int L)
{
    if (T < kBoysTmax) {
        const int k = __double2int_rn(T * kBoysPerUnit);
        const double d = k * (1.0 / kBoysPerUnit) - T;
        const double* r = tab + k * kBoysCols + L;
        double f = __ldg(r + 6);
        f = __ldg(r + 5) + d * (1.0 / 6.0) * f;
        f = __ldg(r + 4) + d * (1.0 / 5.0) * f;
        f = __ldg(r + 3) + d * (1.0 / 4.0) * f;
        f = __ldg(r + 2) + d * (1.0 / 3.0) * f;
        f = __ldg(r + 1) + d * (1.0 / 2.0) * f;
        f = __ldg(r + 0) + d * f;
        double x = 1.0 + d * (1.0 / 6.0);
        x = 1.0 + d * (1.0 / 5.0) * x;
        x = 1.0 + d * (1.0 / 4.0) * x;
        x = 1.0 + d * (1.0 / 3.0) * x;
        x = 1.0 + d * (1.0 / 2.0) * x;
        x = 1.0 + d * x;
        const double e = __ldg(tab + k * kBoysCols + kBoysExpCol) * x;
        F[L] = f;
        for (int m = L - 1; m >= 0; m--) F[m] = (2.0 * T * F[m + 1] + e) * (1.0 / (2 * m + 1));
    } else {
        const double e = exp(-T);
        const double h = 0.5 / T;
        F[0] = 0.88622692545275801365 * rsqrt(T);
        for (int m = 1; m <= L; m++) F[m] = ((2 * m - 1) * F[m - 1] - e) * h;
    }
    for (int m = 0; m <= L; m++) F[m] *= pref;
}

// One shell quartet with the nt threads of a block: primitive loop with the
// vertical recurrence and contraction, program-driven.
__device__ void generic_quartet(const QuartetCtx& q, const FockParams& P, const GenLayout& G, const GenProgram& R,
                                double* sm, int tid, int nt)
{
    double* acc = sm + G.acc_off;
    for (int i = tid; i < G.ne * G.nf; i += nt) acc[i] = 0.0;
    __syncthreads();
    for (int ib = 0; ib < q.nbra; ib++) {
        const double4 xb = load_prim_aux(P.prim, q.bra_off + ib);
        const PrimPair pb = load_prim(P, q.bra_off + ib, xb);
        for (int ik = 0; ik < q.nket; ik++) {
            const double4 xk = load_prim_aux(P.prim, q.ket_off + ik);
            if (!prim_survives(q, xb.z, xk.z, P.prim_limit)) continue;   // the same for every thread
            const PrimPair pk = load_prim(P, q.ket_off + ik, xk);
            const double pq = pb.p + pk.p;
            const double sq = rsqrt(pq);
            const double ipq = sq * sq;
            const double rho = pb.p * pk.p * ipq;
            const double PQx = pb.Px - pk.Px, PQy = pb.Py - pk.Py, PQz = pb.Pz - pk.Pz;
            const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
            const double fp = -pk.p * ipq, fq = pb.p * ipq;
            const double WP[3] = {fp * PQx, fp * PQy, fp * PQz};
            const double WQ[3] = {fq * PQx, fq * PQy, fq * PQz};
            const double PA[3] = {pb.PAx, pb.PAy, pb.PAz};
            const double QC[3] = {pk.PAx, pk.PAy, pk.PAz};
            const double o2p = pb.o2p, o2q = pk.o2p, o2pq = 0.5 * ipq;
            const double rp = pk.p * ipq, rq = pb.p * ipq;
            if (tid == 0) boys_rt(P.boys, T, pb.K * pk.K * sq, sm + G.lvl_off[0], G.lt);
            __syncthreads();
            for (int s = 0; s < R.nstage; s++) {
                const int type = R.stage[3 * s], first = R.stage[3 * s + 1], cnt = R.stage[3 * s + 2];
                if (type == 2) {
                    for (int t = tid; t < cnt; t += nt) {
                        const int4 e = R.ent[first + t];
                        acc[e.x] += sm[e.y];
                    }
                } else {
                    for (int t = tid; t < cnt; t += nt) {
                        const int4 e = R.ent[first + t];
                        const int mt = R.meta[first + t];
                        const int i = mt & 3, mc = (mt >> 2) & 15, mg = (mt >> 6) & 15, nm = mt >> 10;
                        const double* a = sm + e.y;
                        double* o = sm + e.x;
                        const double ci = type == 0 ? PA[i] : QC[i];
                        const double wi = type == 0 ? WP[i] : WQ[i];
                        const double cm = mc * (type == 0 ? o2p : o2q), r = type == 0 ? rp : rq;
                        const double* c = sm + (e.z >= 0 ? e.z : 0);
                        const double* gg = sm + (e.w >= 0 ? e.w : 0);
                        const double gm = mg * o2pq;
                        for (int m = 0; m < nm; m++) {
                            double v = ci * a[m] + wi * a[m + 1];
                            if (e.z >= 0) v += cm * (c[m] - r * c[m + 1]);
                            if (e.w >= 0) v += gm * gg[m + 1];
                            o[m] = v;
                        }
                    }
                }
                __syncthreads();
            }
        }
    }
}

// Horizontal recurrence in closed form (ket side into X, then bra side per
// integral into I) and the Coulomb/exchange contraction into six
// shared-memory blocks, flushed once per quartet with the weights of
// digest_coulomb / digest_exchange.
// The horizontal recurrence of the quartet (its contracted [e0|f0] in acc):
// the ket side into X, then the quartet's integrals I[ab][cd] (component
// order of the basis functions) at G.i_off.  Ends with a barrier.
__device__ void generic_transfer(const QuartetCtx& q, const GenLayout& G, const GenProgram& R, double* sm, int tid,
                                 int nt)
{
    const int na = g_ncart(G.la), nb = g_ncart(G.lb), nc = g_ncart(G.lc), nd = g_ncart(G.ld);
    const int ncd = nc * nd;
    const double* acc = sm + G.acc_off;
    double* X = sm + G.x_off;
    double* pw = sm + G.pw_off;
    if (tid < 24) {
        const double AB[3] = {q.ABx, q.ABy, q.ABz}, CD[3] = {q.CDx, q.CDy, q.CDz};
        const double base = tid < 12 ? AB[tid / 4] : CD[(tid - 12) / 4];
        double v = 1.0;
        for (int k = 0; k < (tid & 3); k++) v *= base;
        pw[tid] = v;
    }
    __syncthreads();
    // ket side: X[e][cd] = sum_k C * CD^pw * acc[e][f]
    for (int t = tid; t < G.ne * ncd; t += nt) {
        const int e = t / ncd, cd = t - e * ncd;
        double v = 0.0;
        for (int j = R.kstart[cd]; j < R.kstart[cd + 1]; j++) {
            const int4 k = R.kterm[j];
            v += k.z * pw[12 + (k.y & 15)] * pw[16 + ((k.y >> 4) & 15)] * pw[20 + (k.y >> 8)] * acc[e * G.nf + k.x];
        }
        X[t] = v;
    }
    __syncthreads();
    const int nab = na * nb, nout = nab * ncd;
    // the quartet's integrals I[ab][cd] (bra side of the horizontal recurrence)
    double* I = sm + G.i_off;
    for (int o = tid; o < nout; o += nt) {
        const int ab = o / ncd, cd = o - ab * ncd;
        double v = 0.0;
        for (int j = R.bstart[ab]; j < R.bstart[ab + 1]; j++) {
            const int4 k = R.bterm[j];
            v += k.z * pw[k.y & 15] * pw[4 + ((k.y >> 4) & 15)] * pw[8 + (k.y >> 8)] * X[k.x * ncd + cd];
        }
        I[o] = v;
    }
    __syncthreads();
}

__device__ void generic_digest(const QuartetCtx& q, const FockParams& P, const GenLayout& G, const GenProgram& R,
                               double* sm, int tid, int nt)
{
    const int na = g_ncart(G.la), nb = g_ncart(G.lb), nc = g_ncart(G.lc), nd = g_ncart(G.ld);
    const int ncd = nc * nd;
    double* Db = sm + G.d_off;
    double* Jb = sm + G.j_off;
    const int o_ab = 0, o_cd = o_ab + na * nb, o_ac = o_cd + nc * nd, o_ad = o_ac + na * nc, o_bc = o_ad + na * nd,
              o_bd = o_bc + nb * nc, nblk = o_bd + nb * nd;
    const double* Dm = P.dense;
    const int n = P.nbasis;
    const int a0 = q.bfA, b0 = q.bfB, c0 = q.bfC, d0 = q.bfD;
    for (int t = tid; t < nblk; t += nt) {
        int r, c;
        if (t < o_cd) r = a0 + (t - o_ab) / nb, c = b0 + (t - o_ab) % nb;
        else if (t < o_ac) r = c0 + (t - o_cd) / nd, c = d0 + (t - o_cd) % nd;
        else if (t < o_ad) r = a0 + (t - o_ac) / nc, c = c0 + (t - o_ac) % nc;
        else if (t < o_bc) r = a0 + (t - o_ad) / nd, c = d0 + (t - o_ad) % nd;
        else if (t < o_bd) r = b0 + (t - o_bc) / nc, c = c0 + (t - o_bc) % nc;
        else r = b0 + (t - o_bd) / nd, c = d0 + (t - o_bd) % nd;
        Db[t] = __ldg(Dm + (size_t)r * n + c);
        Jb[t] = 0.0;
    }
    generic_transfer(q, G, R, sm, tid, nt);   // its first barrier covers the density blocks
    const bool exch = P.hybrid != 0.0;
    const int nab = na * nb;
    const double* I = sm + G.i_off;
    // contraction with the density, one thread per output element of each of
    // the six blocks (no atomics): J_ab = sum_cd D_cd I, J_cd = sum_ab D_ab I,
    // K_ac = sum_bd D_bd I, K_ad = sum_bc D_bc I, K_bc = sum_ad D_ad I,
    // K_bd = sum_ac D_ac I
    for (int t = tid; t < (exch ? nblk : o_ac); t += nt) {
        double v = 0.0;
        if (t < o_cd) {
            const int ab = t - o_ab;
            for (int cd = 0; cd < ncd; cd++) v += Db[o_cd + cd] * I[ab * ncd + cd];
        } else if (t < o_ac) {
            const int cd = t - o_cd;
            for (int ab = 0; ab < nab; ab++) v += Db[o_ab + ab] * I[ab * ncd + cd];
        } else if (t < o_ad) {
            const int ia = (t - o_ac) / nc, ic = (t - o_ac) - ia * nc;
            for (int ib = 0; ib < nb; ib++)
                for (int id = 0; id < nd; id++) v += Db[o_bd + ib * nd + id] * I[(ia * nb + ib) * ncd + ic * nd + id];
        } else if (t < o_bc) {
            const int ia = (t - o_ad) / nd, id = (t - o_ad) - ia * nd;
            for (int ib = 0; ib < nb; ib++)
                for (int ic = 0; ic < nc; ic++) v += Db[o_bc + ib * nc + ic] * I[(ia * nb + ib) * ncd + ic * nd + id];
        } else if (t < o_bd) {
            const int ib = (t - o_bc) / nc, ic = (t - o_bc) - ib * nc;
            for (int ia = 0; ia < na; ia++)
                for (int id = 0; id < nd; id++) v += Db[o_ad + ia * nd + id] * I[(ia * nb + ib) * ncd + ic * nd + id];
        } else {
            const int ib = (t - o_bd) / nd, id = (t - o_bd) - ib * nd;
            for (int ia = 0; ia < na; ia++)
                for (int ic = 0; ic < nc; ic++) v += Db[o_ac + ia * nc + ic] * I[(ia * nb + ib) * ncd + ic * nd + id];
        }
        Jb[t] = v;
    }
    __syncthreads();
    const double wj = 2.0 * q.w, wk = -0.5 * P.hybrid * q.w;
    for (int t = tid; t < (exch ? nblk : o_ac); t += nt) {
        int r, c;
        double wgt;
        if (t < o_cd) r = a0 + (t - o_ab) / nb, c = b0 + (t - o_ab) % nb, wgt = wj;
        else if (t < o_ac) r = c0 + (t - o_cd) / nd, c = d0 + (t - o_cd) % nd, wgt = wj;
        else if (t < o_ad) r = a0 + (t - o_ac) / nc, c = c0 + (t - o_ac) % nc, wgt = wk;
        else if (t < o_bc) r = a0 + (t - o_ad) / nd, c = d0 + (t - o_ad) % nd, wgt = wk;
        else if (t < o_bd) r = b0 + (t - o_bc) / nc, c = c0 + (t - o_bc) % nc, wgt = wk;
        else r = b0 + (t - o_bd) / nd, c = d0 + (t - o_bd) % nd, wgt = wk;
        fock_add(P.fock, n, r, c, wgt * Jb[t], P.fixed_point);
    }
    __syncthreads();
}

// One block per shell quartet (its warps share the recurrence stages and
// the contraction; the shared-memory layout of one quartet bounds the blocks
// per SM, so more threads per quartet is how occupancy grows); fp32_list:
// walk the class's FP32 list (mixed precision) -- these classes compute in
// FP64 either way.
__global__ void __launch_bounds__(256) fock_generic_kernel(const FockParams P, int cls, const GenLayout G,
                                                          const GenProgram R, int fp32_list)
{
    extern __shared__ double sm[];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int n = fp32_list ? P.class_count32[cls] : P.class_count[cls];
    const Quartet* list = fp32_list ? P.quartets + (P.class_end[cls] - n) : P.quartets + P.class_offset[cls];
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        QuartetCtx q;
        load_quartet(P, list[i], true, q);
        generic_quartet(q, P, G, R, sm, tid, nt);
        generic_digest(q, P, G, R, sm, tid, nt);
    }
}

// gpu_aoint_'s counterpart for these classes: the integrals of quartets
// [O.qbegin, O.qend) of the class list, each kept once (aoint_emit), instead
// of their digestion.
__global__ void __launch_bounds__(256) aoint_generic_kernel(const FockParams P, int cls, const GenLayout G,
                                                           const GenProgram R, const AoIntOut O)
{
    extern __shared__ double sm[];
    const int tid = threadIdx.x, nt = blockDim.x;
    const int n = P.class_count[cls];
    const Quartet* list = P.quartets + P.class_offset[cls];
    const long long end = O.qend < n ? O.qend : n;
    const int nb = g_ncart(G.lb), nc = g_ncart(G.lc), nd = g_ncart(G.ld), ncd = nc * nd;
    const int nout = g_ncart(G.la) * nb * ncd;
    for (long long i = O.qbegin + blockIdx.x; i < end; i += gridDim.x) {
        QuartetCtx q;
        load_quartet(P, list[i], true, q);
        generic_quartet(q, P, G, R, sm, tid, nt);
        generic_transfer(q, G, R, sm, tid, nt);
        const double* I = sm + G.i_off;
        for (int o = tid; o < nout; o += nt) {
            const int ab = o / ncd, cd = o - ab * ncd;
            aoint_emit(O, q, q.bfA + ab / nb, q.bfB + ab % nb, q.bfC + cd / nd, q.bfD + cd % nd, I[o]);
        }
        __syncthreads();
    }
}

// Schwarz records of an f pair type (schwarz_kernel's contract): mode 0,
// one warp per (shell pair, sub-shell pair) record with all its primitive
// pairs; mode 1, one warp per primitive pair alone.  The diagonal block
// (ab|ab) comes from the class (LA LB | LA LB) program; the output is
// max over components of |(ab|ab)| cons_a^2 cons_b^2.
__global__ void __launch_bounds__(32) schwarz_generic_kernel(const SchwarzParams S, const FockParams P,
                                                            const GenLayout G, const GenProgram R, int begin,
                                                            int end, int mode)
{
    extern __shared__ double sm[];
    const int lane = threadIdx.x;
    const int na = g_ncart(G.la), nb = g_ncart(G.lb);
    const int p_begin = S.pair_bf[begin].z;
    const int4 last = S.pair_bf[end - 1];
    const int nwork = mode == 0 ? end - begin : last.z + last.w - p_begin;
    for (int w = blockIdx.x; w < nwork; w += gridDim.x) {
        int rec = begin + w, p0 = 0, np = 0;
        if (mode == 0) {
            np = S.pair_bf[rec].w;
        } else {
            const int p = p_begin + w;
            int lo = begin, hi = end - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (S.pair_bf[mid].z <= p) lo = mid; else hi = mid - 1;
            }
            rec = lo;
            p0 = p - S.pair_bf[rec].z;
            np = 1;
        }
        const int4 info = S.pair_bf[rec];
        const double4 ab = S.pair_AB[rec];
        QuartetCtx q{};
        q.active = true;
        q.bra_off = q.ket_off = info.z + p0;
        q.nbra = q.nket = np;
        q.ABx = q.CDx = ab.x;
        q.ABy = q.CDy = ab.y;
        q.ABz = q.CDz = ab.z;
        q.dnmax = 1.0;
        q.swap = false;
        generic_quartet(q, P, G, R, sm, lane, 32);
        double* pw = sm + G.pw_off;
        if (lane < 24) {
            const double base = lane < 12 ? (&ab.x)[lane / 4] : (&ab.x)[(lane - 12) / 4];
            double v = 1.0;
            for (int k = 0; k < (lane & 3); k++) v *= base;
            pw[lane] = v;
        }
        __syncwarp();
        const double* acc = sm + G.acc_off;
        double mx = 0.0;
        for (int o = lane; o < na * nb; o += 32) {
            double v = 0.0;
            for (int jb = R.bstart[o]; jb < R.bstart[o + 1]; jb++) {
                const int4 tb = R.bterm[jb];
                double sk = 0.0;
                for (int jk = R.kstart[o]; jk < R.kstart[o + 1]; jk++) {
                    const int4 tk = R.kterm[jk];
                    sk += tk.z * pw[12 + (tk.y & 15)] * pw[16 + ((tk.y >> 4) & 15)] * pw[20 + (tk.y >> 8)] *
                          acc[tb.x * G.nf + tk.x];
                }
                v += tb.z * pw[tb.y & 15] * pw[4 + ((tb.y >> 4) & 15)] * pw[8 + (tb.y >> 8)] * sk;
            }
            const double ca = S.cons[info.x + o / nb], cb = S.cons[info.y + o % nb];
            mx = fmax(mx, fabs(v) * ca * ca * cb * cb);
        }
#pragma unroll
        for (int k = 16; k > 0; k >>= 1) mx = fmax(mx, __shfl_xor_sync(FULL, mx, k));
        if (lane == 0) {
            if (mode == 0) S.out_contracted[rec] = mx;
            else S.out_prim[p_begin + w] = mx;
        }
        __syncwarp();
    }
}

// ------------------------------------------------------------ launch
// The host-side program of one class, built once per process.
struct GenHost {
    GenLayout G;
    GenProgramHost H;
    size_t bytes = 0;     // its device image, every array 256-byte aligned
};

static size_t up256(size_t x) { return (x + 255) & ~(size_t)255; }

static const GenHost* gen_host(int la, int lb, int lc, int ld, bool grad)
{
    static std::map<int, GenHost> cache;
    const int key = grad ? (1 << 24) + (((la * 8 + lb) * 8 + lc) * 8 + ld) : ((la * 4 + lb) * 4 + lc) * 4 + ld;
    auto it = cache.find(key);
    if (it != cache.end()) return &it->second;
    GenHost h;
    h.G = gen_layout(la, lb, lc, ld);
    gen_program(h.G, h.H, !grad);
    const GenProgramHost& H = h.H;
    h.bytes = up256(H.stage.size() * sizeof(int)) + up256(H.meta.size() * sizeof(int)) +
              up256(H.ent.size() * sizeof(int4)) + up256(H.kterm.size() * sizeof(int4)) +
              up256(H.bterm.size() * sizeof(int4)) + up256(H.kstart.size() * sizeof(int)) +
              up256(H.bstart.size() * sizeof(int));
    return &(cache[key] = std::move(h));
}

// Copies the program into device memory at mem (256-byte aligned, at least
// h.bytes) on stream st and returns the device view of it.
static int gen_place(const GenHost& h, void* mem, cudaStream_t st, GenProgram* R)
{
    char* p = (char*)mem;
    bool ok = true;
    auto put = [&](const void* src, size_t bytes) {
        void* dst = p;
        if (bytes) ok = ok && cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, st) == cudaSuccess;
        p += up256(bytes);
        return dst;
    };
    const GenProgramHost& H = h.H;
    R->stage = (const int*)put(H.stage.data(), H.stage.size() * sizeof(int));
    R->nstage = (int)H.stage.size() / 3;
    R->meta = (const int*)put(H.meta.data(), H.meta.size() * sizeof(int));
    R->ent = (const int4*)put(H.ent.data(), H.ent.size() * sizeof(int4));
    R->kterm = (const int4*)put(H.kterm.data(), H.kterm.size() * sizeof(int4));
    R->bterm = (const int4*)put(H.bterm.data(), H.bterm.size() * sizeof(int4));
    R->kstart = (const int*)put(H.kstart.data(), H.kstart.size() * sizeof(int));
    R->bstart = (const int*)put(H.bstart.data(), H.bstart.size() * sizeof(int));
    return ok ? 0 : -1;
}

struct GenCached {
    GenLayout G;
    GenProgram R;
    void* mem = nullptr;
    int dev = -1;
};

// grad: the layout and recurrence program of the extended range of the
// gradient kernel (shells may exceed f; no horizontal terms).  The device
// copy lives in memory of its own, one per class and device.
static GenCached* gen_cached(int la, int lb, int lc, int ld, bool grad = false)
{
    static std::map<int, GenCached> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    const int key = grad ? (1 << 24) + (((la * 8 + lb) * 8 + lc) * 8 + ld) + 4096 * dev
                         : ((la * 4 + lb) * 4 + lc) * 4 + ld + 256 * dev;
    auto it = cache.find(key);
    if (it != cache.end()) return &it->second;
    const GenHost* h = gen_host(la, lb, lc, ld, grad);
    GenCached c;
    c.G = h->G;
    if (cudaMalloc(&c.mem, h->bytes) != cudaSuccess) return nullptr;
    if (gen_place(*h, c.mem, 0, &c.R) != 0 || cudaStreamSynchronize(0) != cudaSuccess) {
        cudaFree(c.mem);
        return nullptr;
    }
    c.dev = dev;
    return &(cache[key] = c);
}

size_t generic_program_bytes(int la, int lb, int lc, int ld) { return gen_host(la, lb, lc, ld, false)->bytes; }

// Shared-memory bytes, opt-in attribute and grid of one generic launch.
static int generic_launch_shape(const GenLayout& G, int nq, int nsm, int* nt_out, size_t* bytes_out, int* grid_out)
{
    const size_t bytes = (size_t)G.total * sizeof(double);
    int dev = 0, maxsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (bytes > (size_t)maxsm) return -1;
    static int configured = 0;
    if (bytes > 48 * 1024 && configured < maxsm) {
        if (cudaFuncSetAttribute(fock_generic_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm) !=
            cudaSuccess)
            return -1;
        configured = maxsm;
    }
    // threads per quartet (QB_GEN_THREADS, default 128)
    static const int nt = [] {
        const char* e = getenv("QB_GEN_THREADS");
        const int v = e ? atoi(e) : 128;
        return (v == 32 || v == 64 || v == 128 || v == 256) ? v : 128;
    }();
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fock_generic_kernel, nt, bytes);
    *nt_out = nt;
    *bytes_out = bytes;
    *grid_out = std::max(1, std::min(nq, nsm * std::max(per_sm, 1)));
    return 0;
}

// launch_generic_class with the class program copied into caller memory
// (mem, 256-byte aligned, at least generic_program_bytes of the class) on
// the launch stream instead of memory of its own: allocates nothing.
int launch_generic_class_placed(int cls, int la, int lb, int lc, int ld, const FockParams& P, int nq, int nsm,
                                void* mem, size_t cap, cudaStream_t st)
{
    if (nq <= 0) return 0;
    const GenHost* h = gen_host(la, lb, lc, ld, false);
    if (h->bytes > cap) return -2;
    int nt = 0, grid = 0;
    size_t bytes = 0;
    if (generic_launch_shape(h->G, nq, nsm, &nt, &bytes, &grid)) return -1;
    GenProgram R;
    if (gen_place(*h, mem, st, &R)) return -3;
    QB_LAUNCH(fock_generic_kernel, grid, nt, bytes, st, P, cls, h->G, R, 0);
    return nt;
}

int launch_generic_class(int cls, int la, int lb, int lc, int ld, const FockParams& P, int nq, int nsm, int fp32_list,
                         cudaStream_t st)
{
    if (nq <= 0) return 0;
    const GenCached* gc = gen_cached(la, lb, lc, ld);
    if (!gc) return -1;
    int nt = 0, grid = 0;
    size_t bytes = 0;
    if (generic_launch_shape(gc->G, nq, nsm, &nt, &bytes, &grid)) return -1;
    QB_LAUNCH(fock_generic_kernel, grid, nt, bytes, st, P, cls, gc->G, gc->R, fp32_list);
    return nt;
}

// The stored-integral kernel of a generic class over the slice of O.
int launch_generic_store(int cls, int la, int lb, int lc, int ld, const FockParams& P, const AoIntOut& O, int nsm,
                         cudaStream_t st)
{
    const long long nq = O.qend - O.qbegin;
    if (nq <= 0) return 0;
    const GenCached* gc = gen_cached(la, lb, lc, ld);
    if (!gc) return -1;
    int nt = 0, grid = 0;
    size_t bytes = 0;
    if (generic_launch_shape(gc->G, (int)std::min<long long>(nq, 1 << 30), nsm, &nt, &bytes, &grid)) return -1;
    int dev = 0, maxsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    static int configured = 0;
    if (bytes > 48 * 1024 && configured < maxsm) {
        if (cudaFuncSetAttribute(aoint_generic_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm) !=
            cudaSuccess)
            return -1;
        configured = maxsm;
    }
    QB_LAUNCH(aoint_generic_kernel, grid, nt, bytes, st, P, cls, gc->G, gc->R, O);
    return nt;
}

int launch_generic_schwarz(int la, int lb, const SchwarzParams& S, int begin, int end, int mode, int nsm,
                           cudaStream_t st)
{
    if (end <= begin) return 0;
    const GenCached* gc = gen_cached(la, lb, la, lb);
    if (!gc) return -1;
    const size_t bytes = (size_t)gc->G.total * sizeof(double);
    int dev = 0, maxsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (bytes > (size_t)maxsm) return -1;
    if (bytes > 48 * 1024 &&
        cudaFuncSetAttribute(schwarz_generic_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, maxsm) != cudaSuccess)
        return -1;
    FockParams P{};
    P.prim = S.prim;
    P.boys = S.boys;
    P.prim_limit = -1.0;   // every primitive pair counts in the bound
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, schwarz_generic_kernel, 32, bytes);
    const int grid = std::max(1, nsm * std::max(per_sm, 1));
    QB_LAUNCH(schwarz_generic_kernel, grid, 32, bytes, st, S, P, gc->G, gc->R, begin, end, mode);
    return 0;
}

size_t generic_class_smem(int la, int lb, int lc, int ld)
{
    return (size_t)gen_layout(la, lb, lc, ld).total * sizeof(double);
}

// ------------------------------------------------------------ gradient
// Two-electron gradient of the classes with an f shell (no straight-line
// gradient kernels exist for them): one 128-thread block per shell quartet.
// The vertical recurrence of the class extended by one unit on each side,
// [e0|f0] with |e| <= LA+LB+1, |f| <= LC+LD+1 (the program of gen_program for
// that range), is contracted over the primitive quartets into four sums with
// the weights 1, 2 alpha, 2 beta and 2 gamma (the exponents of A, B and C);
// then per integral and direction, by the horizontal transfer in closed form
// on both sides,
//   d/dA_i (ab|cd) = 2 alpha (a+1_i b|cd) - a_i (a-1_i b|cd),
//   d/dB_i (ab|cd) = 2 beta  (a b+1_i|cd) - b_i (a b-1_i|cd),
//   d/dC_i (ab|cd) = 2 gamma (ab|c+1_i d) - c_i (ab|c-1_i d),
// contracted with the density products of the generated gradient kernels
// (4 D_ab D_cd - h (D_ac D_bd + D_ad D_bc)), D by translational invariance.
// The recurrence buffers and sums of the extended range exceed shared memory
// for the large classes, so each block works in its own slice of a global
// scratch array (L2-resident for all but the largest classes).
__constant__ int kQuickCartD[4][10][3] = {
    {{0, 0, 0}},
    {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}},
    {{2, 0, 0}, {1, 1, 0}, {0, 2, 0}, {1, 0, 1}, {0, 1, 1}, {0, 0, 2}},
    {{3, 0, 0}, {2, 1, 0}, {1, 2, 0}, {0, 3, 0}, {2, 0, 1}, {1, 1, 1}, {0, 2, 1}, {1, 0, 2}, {0, 1, 2}, {0, 0, 3}},
};

struct GenGradInfo {
    int la, lb, lc, ld;     // the class
    int elo, flo;           // lowest |e|, |f| held in the sums
    int ne, nf;             // extents of the sums (rows |e| in [elo, LA+LB+1], columns |f| in [flo, LC+LD+1])
    long long per_block;    // scratch doubles per block
    long long x_off[5];     // ket-transformed sums: 2a (c,d), 1 (c,d), 2b (c,d), 2g (c+1,d), 1 (c-1,d)
    int fp32_list;          // walk the class's FP32 list of the mixed split (evaluated in FP64 here)
    long long y_off[6];     // both sides transferred: (a+1 b|, (a-1 b|, (a b+1|, (a b-1|, |c+1 d), |c-1 d)
};

__device__ __forceinline__ int gen_gidx(int x, int y, int z, int lo)
{
    const int n = x + y + z, t = y + z;
    return g_ncum(n - 1) - g_ncum(lo - 1) + t * (t + 1) / 2 + z;
}

// C(n, k) for 0 <= k <= n <= 5 from two immediates (rows packed 4 bits per
// entry, entry n(n+1)/2 + k): the lanes of a warp ask for different entries,
// which a __constant__ table would serve one address at a time.
__device__ __forceinline__ int binom5(int n, int k)
{
    constexpr unsigned long long lo = 0x146411331121111ull;   // entries 0..14
    constexpr unsigned long long hi = 0x15aa51ull;              // entries 15..20
    const int idx = n * (n + 1) / 2 + k;
    return idx < 15 ? (int)((lo >> (4 * idx)) & 15ull) : (int)((hi >> (4 * (idx - 15))) & 15ull);
}

// canonical index of (x, y, z) inside its shell, and back
__device__ __forceinline__ int gen_canon(int y, int z) { const int t = y + z; return t * (t + 1) / 2 + z; }
__device__ __forceinline__ void gen_uncanon(int l, int idx, int* e)
{
    int t = 0;
    while ((t + 1) * (t + 2) / 2 <= idx) t++;
    e[2] = idx - t * (t + 1) / 2;
    e[1] = t - e[2];
    e[0] = l - t;
}

// X[row][c d] = sum_kd C(d,kd) CD^(d-kd) E[row][c+kd] for every row of the
// sums, c in shell lcx, d in shell ld (canonical order).  CDp[3][8]: powers.
__device__ void gen_ket_transform(const double* E, double* X, const GenGradInfo& I, int lcx, int ldx,
                                  const double* CDp, int tid, int nt)
{
    const int ncx = g_ncart(lcx), ndx = g_ncart(ldx), cols = ncx * ndx;
    for (int t = tid; t < I.ne * cols; t += nt) {
        const int row = t / cols, col = t - row * cols;
        int c[3], d[3];
        gen_uncanon(lcx, col / ndx, c);
        gen_uncanon(ldx, col % ndx, d);
        const double* Er = E + (size_t)row * I.nf;
        double v = 0.0;
        for (int kx = 0; kx <= d[0]; kx++)
            for (int ky = 0; ky <= d[1]; ky++)
                for (int kz = 0; kz <= d[2]; kz++)
                    v += binom5(d[0], kx) * binom5(d[1], ky) * binom5(d[2], kz) * CDp[d[0] - kx] *
                         CDp[8 + d[1] - ky] * CDp[16 + d[2] - kz] * Er[gen_gidx(c[0] + kx, c[1] + ky, c[2] + kz, I.flo)];
        X[t] = v;
    }
}

// sum_kb C(b,kb) AB^(b-kb) X[a+kb][col]
__device__ __forceinline__ double gen_bra_sum(const double* X, int cols, int col, const int* a, const int* b,
                                              const GenGradInfo& I, const double* ABp)
{
    double s = 0.0;
    for (int kx = 0; kx <= b[0]; kx++)
        for (int ky = 0; ky <= b[1]; ky++)
            for (int kz = 0; kz <= b[2]; kz++)
                s += binom5(b[0], kx) * binom5(b[1], ky) * binom5(b[2], kz) * ABp[b[0] - kx] * ABp[8 + b[1] - ky] *
                     ABp[16 + b[2] - kz] * X[(size_t)gen_gidx(a[0] + kx, a[1] + ky, a[2] + kz, I.elo) * cols + col];
    return s;
}

// Y[a'][b'][col] = bra transfer of X for every a' in shell lax, b' in shell
// lbx and ket column col (canonical orders), the block's threads sharing it.
__device__ void gen_bra_table(const double* X, int cols, int lax, int lbx, double* Y, const GenGradInfo& I,
                              const double* ABp, int tid, int nt)
{
    const int nax = g_ncart(lax), nbx = g_ncart(lbx);
    for (int t = tid; t < nax * nbx * cols; t += nt) {
        const int col = t % cols, r = t / cols;
        int a[3], b[3];
        gen_uncanon(lax, r / nbx, a);
        gen_uncanon(lbx, r % nbx, b);
        Y[t] = gen_bra_sum(X, cols, col, a, b, I, ABp);
    }
}

__global__ void __launch_bounds__(128) grad_generic_kernel(const FockParams P, const GradExtra X, int cls,
                                                          const GenLayout G, const GenProgram R, const GenGradInfo I,
                                                          double* scratch)
{
    const int tid = threadIdx.x, nt = blockDim.x;
    double* sm = scratch + (size_t)blockIdx.x * I.per_block;   // this block's recurrence buffers and sums
    const size_t nacc = (size_t)I.ne * I.nf;
    double* E1 = sm + G.acc_off;
    double* Ea = sm + G.total;
    double* Eb = Ea + nacc;
    double* Ec = Eb + nacc;
    __shared__ double red[9][4];
    // QUICK's Cartesian orders in shared memory: the lanes of a warp read
    // different entries, which a __constant__ table serves one at a time
    __shared__ int sCart[4 * 10 * 3];
    for (int i = tid; i < 4 * 10 * 3; i += nt) sCart[i] = (&kQuickCartD[0][0][0])[i];
    const int na = g_ncart(I.la), nb = g_ncart(I.lb), nc = g_ncart(I.lc), nd = g_ncart(I.ld);
    const int n = I.fp32_list ? P.class_count32[cls] : P.class_count[cls];
    const Quartet* list = I.fp32_list ? P.quartets + (P.class_end[cls] - n) : P.quartets + P.class_offset[cls];
    for (int qi = blockIdx.x; qi < n; qi += gridDim.x) {
        QuartetCtx q;
        load_quartet(P, list[qi], true, q);
        for (size_t i = tid; i < nacc; i += nt) E1[i] = Ea[i] = Eb[i] = Ec[i] = 0.0;
        __syncthreads();
        for (int ib = 0; ib < q.nbra; ib++) {
            const double4 xb = load_prim_aux(P.prim, q.bra_off + ib);
            const PrimPair pb = load_prim(P, q.bra_off + ib, xb);
            for (int ik = 0; ik < q.nket; ik++) {
                const double4 xk = load_prim_aux(P.prim, q.ket_off + ik);
                if (!prim_survives(q, xb.z, xk.z, P.prim_limit)) continue;   // the same for every thread
                const PrimPair pk = load_prim(P, q.ket_off + ik, xk);
                const double pq = pb.p + pk.p;
                const double sq = rsqrt(pq);
                const double ipq = sq * sq;
                const double rho = pb.p * pk.p * ipq;
                const double PQx = pb.Px - pk.Px, PQy = pb.Py - pk.Py, PQz = pb.Pz - pk.Pz;
                const double T = rho * (PQx * PQx + PQy * PQy + PQz * PQz);
                const double fp = -pk.p * ipq, fq = pb.p * ipq;
                const double WP[3] = {fp * PQx, fp * PQy, fp * PQz};
                const double WQ[3] = {fq * PQx, fq * PQy, fq * PQz};
                const double PA[3] = {pb.PAx, pb.PAy, pb.PAz};
                const double QC[3] = {pk.PAx, pk.PAy, pk.PAz};
                const double o2p = pb.o2p, o2q = pk.o2p, o2pq = 0.5 * ipq;
                const double rp = pk.p * ipq, rq = pb.p * ipq;
                // exponent weights of the derivative sums: 2 alpha, 2 beta, 2 gamma
                const double wa = 2.0 * xb.y, wb = 2.0 * (pb.p - xb.y), wc = 2.0 * xk.y;
                if (tid == 0) boys_rt(P.boys, T, pb.K * pk.K * sq, sm + G.lvl_off[0], G.lt);
                __syncthreads();
                for (int s = 0; s < R.nstage; s++) {
                    const int type = R.stage[3 * s], first = R.stage[3 * s + 1], cnt = R.stage[3 * s + 2];
                    if (type == 2) {
                        for (int t = tid; t < cnt; t += nt) {
                            const int4 e = R.ent[first + t];
                            const double v = sm[e.y];
                            E1[e.x] += v;
                            Ea[e.x] += wa * v;
                            Eb[e.x] += wb * v;
                            Ec[e.x] += wc * v;
                        }
                    } else {
                        for (int t = tid; t < cnt; t += nt) {
                            const int4 e = R.ent[first + t];
                            const int mt = R.meta[first + t];
                            const int i = mt & 3, mc = (mt >> 2) & 15, mg = (mt >> 6) & 15, nm = mt >> 10;
                            const double* a = sm + e.y;
                            double* o = sm + e.x;
                            const double ci = type == 0 ? PA[i] : QC[i];
                            const double wi = type == 0 ? WP[i] : WQ[i];
                            const double cm = mc * (type == 0 ? o2p : o2q), r = type == 0 ? rp : rq;
                            const double* c = sm + (e.z >= 0 ? e.z : 0);
                            const double* gg = sm + (e.w >= 0 ? e.w : 0);
                            const double gm = mg * o2pq;
                            for (int m = 0; m < nm; m++) {
                                double v = ci * a[m] + wi * a[m + 1];
                                if (e.z >= 0) v += cm * (c[m] - r * c[m + 1]);
                                if (e.w >= 0) v += gm * gg[m + 1];
                                o[m] = v;
                            }
                        }
                    }
                    __syncthreads();
                }
            }
        }
        // derivative integrals contracted with the density products: the ket
        // side of the transfer once per sum, then short bra sums per integral
        __shared__ double ABp[24], CDp[24];
        if (tid < 48) {
            const double base = tid < 24 ? (tid < 8 ? q.ABx : (tid < 16 ? q.ABy : q.ABz))
                                         : (tid < 32 ? q.CDx : (tid < 40 ? q.CDy : q.CDz));
            double v = 1.0;
            for (int k = 0; k < (tid & 7); k++) v *= base;
            if (tid < 24) ABp[tid] = v;
            else CDp[tid - 24] = v;
        }
        __syncthreads();
        double* XA = sm + I.x_off[0];
        double* X1 = sm + I.x_off[1];
        double* XB = sm + I.x_off[2];
        double* XCp = sm + I.x_off[3];
        double* XCm = sm + I.x_off[4];
        gen_ket_transform(Ea, XA, I, I.lc, I.ld, CDp, tid, nt);
        gen_ket_transform(E1, X1, I, I.lc, I.ld, CDp, tid, nt);
        gen_ket_transform(Eb, XB, I, I.lc, I.ld, CDp, tid, nt);
        gen_ket_transform(Ec, XCp, I, I.lc + 1, I.ld, CDp, tid, nt);
        if (I.lc > 0) gen_ket_transform(E1, XCm, I, I.lc - 1, I.ld, CDp, tid, nt);
        __syncthreads();
        // bra side of the transfer once per (a', b') and ket column: the
        // derivative integrals of every output then read these tables
        const int na_ = g_ncart(I.la), nb_ = g_ncart(I.lb), nc_ = g_ncart(I.lc), nd_ = g_ncart(I.ld);
        const int ccd = nc_ * nd_, ccp = g_ncart(I.lc + 1) * nd_, ccm = g_ncart(I.lc - 1) * nd_;
        double* YA = sm + I.y_off[0];
        double* Y1a = sm + I.y_off[1];
        double* YB = sm + I.y_off[2];
        double* Y1b = sm + I.y_off[3];
        double* YCp = sm + I.y_off[4];
        double* YCm = sm + I.y_off[5];
        gen_bra_table(XA, ccd, I.la + 1, I.lb, YA, I, ABp, tid, nt);
        if (I.la > 0) gen_bra_table(X1, ccd, I.la - 1, I.lb, Y1a, I, ABp, tid, nt);
        gen_bra_table(XB, ccd, I.la, I.lb + 1, YB, I, ABp, tid, nt);
        if (I.lb > 0) gen_bra_table(X1, ccd, I.la, I.lb - 1, Y1b, I, ABp, tid, nt);
        gen_bra_table(XCp, ccp, I.la, I.lb, YCp, I, ABp, tid, nt);
        if (I.lc > 0) gen_bra_table(XCm, ccm, I.la, I.lb, YCm, I, ABp, tid, nt);
        __syncthreads();
        const double* Dm = P.dense;
        const int nbf = P.nbasis;
        const double hx = P.hybrid;
        const int nbp = g_ncart(I.lb + 1), nbm = g_ncart(I.lb - 1);
        double gs[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
        const int nout = na_ * nb_ * nc_ * nd_;
        for (int o = tid; o < nout; o += nt) {
            int r = o;
            const int id = r % nd_; r /= nd_;
            const int ic = r % nc_; r /= nc_;
            const int ibb = r % nb_; r /= nb_;
            const int ia = r;
            int a[3], b[3], c[3], d[3];
            for (int k = 0; k < 3; k++) {
                a[k] = sCart[(I.la * 10 + ia) * 3 + k];
                b[k] = sCart[(I.lb * 10 + ibb) * 3 + k];
                c[k] = sCart[(I.lc * 10 + ic) * 3 + k];
                d[k] = sCart[(I.ld * 10 + id) * 3 + k];
            }
            const int fa = q.bfA + ia, fb = q.bfB + ibb, fc = q.bfC + ic, fd = q.bfD + id;
            const double Dab = __ldg(Dm + (size_t)fa * nbf + fb), Dcd = __ldg(Dm + (size_t)fc * nbf + fd);
            const double Dac = __ldg(Dm + (size_t)fa * nbf + fc), Dbd = __ldg(Dm + (size_t)fb * nbf + fd);
            const double Dad = __ldg(Dm + (size_t)fa * nbf + fd), Dbc = __ldg(Dm + (size_t)fb * nbf + fc);
            const double g = 4.0 * Dab * Dcd - hx * (Dac * Dbd + Dad * Dbc);
            if (g == 0.0) continue;
            const int ca = gen_canon(a[1], a[2]), cb = gen_canon(b[1], b[2]);
            const int dcan = gen_canon(d[1], d[2]);
            const int colcd = gen_canon(c[1], c[2]) * nd_ + dcan;
            for (int i = 0; i < 3; i++) {
                int u[3] = {a[0], a[1], a[2]};
                u[i]++;
                double dA = YA[((size_t)gen_canon(u[1], u[2]) * nb_ + cb) * ccd + colcd];
                if (a[i] > 0) {
                    u[i] -= 2;
                    dA -= a[i] * Y1a[((size_t)gen_canon(u[1], u[2]) * nb_ + cb) * ccd + colcd];
                }
                int v[3] = {b[0], b[1], b[2]};
                v[i]++;
                double dB = YB[((size_t)ca * nbp + gen_canon(v[1], v[2])) * ccd + colcd];
                if (b[i] > 0) {
                    v[i] -= 2;
                    dB -= b[i] * Y1b[((size_t)ca * nbm + gen_canon(v[1], v[2])) * ccd + colcd];
                }
                int w[3] = {c[0], c[1], c[2]};
                w[i]++;
                double dC = YCp[((size_t)ca * nb_ + cb) * ccp + gen_canon(w[1], w[2]) * nd_ + dcan];
                if (c[i] > 0) {
                    w[i] -= 2;
                    dC -= c[i] * YCm[((size_t)ca * nb_ + cb) * ccm + gen_canon(w[1], w[2]) * nd_ + dcan];
                }
                gs[i] += g * dA;
                gs[3 + i] += g * dB;
                gs[6 + i] += g * dC;
            }
        }
        // block sum of the nine components
        const int lane = tid & 31, wid = tid >> 5;
        for (int k = 0; k < 9; k++) {
            double x = gs[k];
            for (int off = 16; off > 0; off >>= 1) x += __shfl_xor_sync(0xffffffffu, x, off);
            if (lane == 0) red[k][wid] = x;
        }
        __syncthreads();
        if (tid == 0) {
            double tot[9];
            for (int k = 0; k < 9; k++) {
                tot[k] = 0.0;
                for (int w2 = 0; w2 < (nt >> 5); w2++) tot[k] += red[k][w2];
            }
            const int4 bs = __ldg(X.pair_sh + q.bra), ks = __ldg(X.pair_sh + q.ket);
            const int A = __ldg(X.shell_atom + bs.x), B = __ldg(X.shell_atom + bs.y);
            const int C = __ldg(X.shell_atom + ks.x), D = __ldg(X.shell_atom + ks.y);
            if (!(A == B && A == C && A == D)) {   // translational invariance: sums to zero
                for (int i = 0; i < 3; i++) {
                    atomicAdd(X.grad + 3 * A + i, q.w * tot[i]);
                    atomicAdd(X.grad + 3 * B + i, q.w * tot[3 + i]);
                    atomicAdd(X.grad + 3 * C + i, q.w * tot[6 + i]);
                    atomicAdd(X.grad + 3 * D + i, -q.w * (tot[i] + tot[3 + i] + tot[6 + i]));
                }
            }
        }
        __syncthreads();
    }
}

static void* g_grad_scratch = nullptr;
static size_t g_grad_scratch_bytes = 0;

void generic_release()
{
    if (g_grad_scratch) cudaFree(g_grad_scratch);
    g_grad_scratch = nullptr;
    g_grad_scratch_bytes = 0;
}

int launch_generic_grad_class(int cls, int la, int lb, int lc, int ld, const FockParams& P, const GradExtra& X, int nq,
                              int nsm, int fp32_list, cudaStream_t st)
{
    if (nq <= 0) return 0;
    const int elo = la > 0 ? la - 1 : 0, flo = lc > 0 ? lc - 1 : 0;
    const GenCached* gc = gen_cached(elo, la + lb + 1 - elo, flo, lc + ld + 1 - flo, true);
    if (!gc) return -1;
    GenGradInfo I{la, lb, lc, ld, elo, flo, gc->G.ne, gc->G.nf, 0, {0, 0, 0, 0, 0}, fp32_list, {0, 0, 0, 0, 0, 0}};
    const long long nacc = (long long)I.ne * I.nf, ndd = g_ncart(ld);
    const long long cols[5] = {g_ncart(lc) * ndd, g_ncart(lc) * ndd, g_ncart(lc) * ndd, g_ncart(lc + 1) * ndd,
                               g_ncart(lc - 1) * ndd};
    long long off = (long long)gc->G.total + 3 * nacc;
    for (int k = 0; k < 5; k++) {
        I.x_off[k] = off;
        off += (long long)I.ne * cols[k];
    }
    const long long na = g_ncart(la), nb = g_ncart(lb);
    const long long ny[6] = {g_ncart(la + 1) * nb * cols[0], g_ncart(la - 1) * nb * cols[0],
                             na * g_ncart(lb + 1) * cols[0], na * g_ncart(lb - 1) * cols[0], na * nb * cols[3],
                             na * nb * cols[4]};
    for (int k = 0; k < 6; k++) {
        I.y_off[k] = off;
        off += ny[k];
    }
    I.per_block = off;
    // scratch of at most 256 MB: four blocks per SM where it allows
    const long long budget = (256LL << 20) / (long long)sizeof(double);
    const long long grid = std::max(1LL, std::min<long long>({(long long)nq, 4LL * nsm, budget / I.per_block}));
    const size_t need = (size_t)grid * (size_t)I.per_block * sizeof(double);
    if (need > g_grad_scratch_bytes) {
        generic_release();
        if (cudaMalloc(&g_grad_scratch, need) != cudaSuccess) {
            g_grad_scratch = nullptr;
            return -1;
        }
        g_grad_scratch_bytes = need;
    }
    QB_LAUNCH(grad_generic_kernel, (int)grid, 128, 0, st, P, X, cls, gc->G, gc->R, I, (double*)g_grad_scratch);
    return 128;
}

}  // namespace qb
