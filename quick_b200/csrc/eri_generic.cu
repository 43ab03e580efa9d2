// Angular classes with an f shell (any shell up to L = 3): one warp per
// shell quartet, the recurrences in shared memory.
//
// The straight-line generated kernels (gen_eri.py) cover s, p and d; their
// f counterparts would be tens of thousands of statements per class.  This
// kernel runs the same algorithm with loops instead:
//
//  * F_m(T), m = 0..LA+LB+LC+LD (lane 0, the table scheme of boys<L>);
//  * the Obara-Saika vertical recurrence [e0|f0]^(m), |e| <= LA+LB,
//    |f| <= LC+LD, one level of |f| at a time (three levels kept), the lanes
//    of the warp sharing each level's entries;
//  * contraction of [e0|f0]^(0) for LA <= |e|, LC <= |f| over the primitive
//    quartets that pass QUICK's primitive screen;
//  * the horizontal recurrence in closed form,
//    (a b| = sum_k prod_i C(b_i, k_i) AB_i^(b_i - k_i) (a + k, 0|, on both sides;
//  * the Coulomb/exchange digestion into six shared-memory blocks, flushed to
//    the Fock matrix once per quartet with the weights of the generated
//    kernels (digest_coulomb / digest_exchange).
//
// QUICK's own spdf path (gpu_get2e_subs.h:413-850 with int.h's
// vertical_spdf* and the 84 x 84 `store`) computes the same integrals.
#include <algorithm>

#include "eri_common.cuh"
#include "qb_internal.h"

namespace qb {

constexpr int kGenMaxL = 3;

__host__ __device__ constexpr int g_ncart(int l) { return l < 0 ? 0 : (l + 1) * (l + 2) / 2; }
// number of Cartesians of all levels <= l
__host__ __device__ constexpr int g_ncum(int l) { return l < 0 ? 0 : (l + 1) * (l + 2) * (l + 3) / 6; }

// position of (x, y, z) inside its level (x descending, then y descending)
__device__ __forceinline__ int g_lidx(int x, int y, int z)
{
    const int t = (x + y + z) - x;
    (void)y;
    return t * (t + 1) / 2 + z;
}
__device__ __forceinline__ void g_cart(int l, int idx, int& x, int& y, int& z)
{
    int t = 0;
    while ((t + 1) * (t + 2) / 2 <= idx) t++;
    z = idx - t * (t + 1) / 2;
    x = l - t;
    y = t - z;
}

// QUICK's Cartesian order of a shell's components (basis.f90:546-643)
__constant__ signed char c_quick_cart[4][10][3] = {
    {{0, 0, 0}},
    {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}},
    {{2, 0, 0}, {1, 1, 0}, {0, 2, 0}, {1, 0, 1}, {0, 1, 1}, {0, 0, 2}},
    {{3, 0, 0}, {2, 1, 0}, {1, 2, 0}, {0, 3, 0}, {2, 0, 1}, {1, 1, 1}, {0, 2, 1}, {1, 0, 2}, {0, 1, 2}, {0, 0, 3}},
};

// Shared-memory layout of one class (doubles), computed on the host.
struct GenLayout {
    int la, lb, lc, ld;
    int lab, lcd, lt;
    int level_size[13];   // entries of VRR level k = |f| (all e, all m)
    int lvl_off[3];       // three rotating level buffers
    int acc_off, ne, nf;  // contracted [e0|f0], |e| in [la, lab], |f| in [lc, lcd]
    int f_off;            // F_m
    int d_off;            // six density blocks
    int j_off;            // six accumulator blocks
    int total;
};

// entries of level k: for every f of the level, for every |e| = l <= lab,
// ncart(l) x (lt - l - k + 1) values of m
static int gen_level_size(int lab, int lt, int k)
{
    int per_f = 0;
    for (int l = 0; l <= lab; l++) per_f += g_ncart(l) * std::max(0, lt - l - k + 1);
    return per_f * g_ncart(k);
}

static GenLayout gen_layout(int la, int lb, int lc, int ld)
{
    GenLayout G{};
    G.la = la; G.lb = lb; G.lc = lc; G.ld = ld;
    G.lab = la + lb;
    G.lcd = lc + ld;
    G.lt = G.lab + G.lcd;
    int mx = 0;
    for (int k = 0; k <= G.lcd; k++) {
        G.level_size[k] = gen_level_size(G.lab, G.lt, k);
        mx = std::max(mx, G.level_size[k]);
    }
    int off = 0;
    for (int j = 0; j < 3; j++) G.lvl_off[j] = off, off += mx;
    G.ne = g_ncum(G.lab) - g_ncum(la - 1);
    G.nf = g_ncum(G.lcd) - g_ncum(lc - 1);
    G.acc_off = off;
    off += G.ne * G.nf;
    G.f_off = off;
    off += G.lt + 8;
    const int na = g_ncart(la), nb = g_ncart(lb), nc = g_ncart(lc), nd = g_ncart(ld);
    const int blocks = na * nb + nc * nd + na * nc + na * nd + nb * nc + nb * nd;
    G.d_off = off;
    off += blocks;
    G.j_off = off;
    off += blocks;
    G.total = off;
    return G;
}

// offset of the (e, m = 0) entry of level k inside one f's block, for e of
// level l at position idx: sum_{j<l} ncart(j)(lt - j - k + 1) + idx (lt - l - k + 1)
__device__ __forceinline__ int g_eoff(const GenLayout& G, int k, int l, int idx)
{
    int off = 0;
    for (int j = 0; j < l; j++) off += g_ncart(j) * (G.lt - j - k + 1);
    return off + idx * (G.lt - l - k + 1);
}
__device__ __forceinline__ int g_fblock(const GenLayout& G, int k)
{
    return G.level_size[k] / g_ncart(k);
}

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

__device__ __forceinline__ double ipow(double x, int n)
{
    double r = 1.0;
    for (int i = 0; i < n; i++) r *= x;
    return r;
}
__device__ __forceinline__ double binom(int n, int k)
{
    double r = 1.0;
    for (int i = 1; i <= k; i++) r = r * (n - k + i) / i;
    return r;
}

// One shell quartet with the 32 lanes of a warp.
__device__ void generic_quartet(const QuartetCtx& q, const FockParams& P, const GenLayout& G, double* sm, int lane)
{
    const int lab = G.lab, lt = G.lt;
    double* acc = sm + G.acc_off;
    double* F = sm + G.f_off;
    for (int i = lane; i < G.ne * G.nf; i += 32) acc[i] = 0.0;
    __syncwarp();
    for (int ib = 0; ib < q.nbra; ib++) {
        const double4 xb = load_prim_aux(P.prim, q.bra_off + ib);
        const PrimPair pb = load_prim(P, q.bra_off + ib, xb);
        for (int ik = 0; ik < q.nket; ik++) {
            const double4 xk = load_prim_aux(P.prim, q.ket_off + ik);
            if (!prim_survives(q, xb.z, xk.z, P.prim_limit)) continue;   // the same for every lane
            const PrimPair pk = load_prim(P, q.ket_off + ik, xk);
            const double pq = pb.p + pk.p;
            const double sq = rsqrt(pq);
            const double ipq = sq * sq;
            const double rho = pb.p * pk.p * ipq;
            const double PQ[3] = {pb.Px - pk.Px, pb.Py - pk.Py, pb.Pz - pk.Pz};
            const double T = rho * (PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2]);
            const double WP[3] = {-pk.p * ipq * PQ[0], -pk.p * ipq * PQ[1], -pk.p * ipq * PQ[2]};
            const double WQ[3] = {pb.p * ipq * PQ[0], pb.p * ipq * PQ[1], pb.p * ipq * PQ[2]};
            const double PA[3] = {pb.PAx, pb.PAy, pb.PAz};
            const double QC[3] = {pk.PAx, pk.PAy, pk.PAz};
            const double o2p = pb.o2p, o2q = pk.o2p, o2pq = 0.5 * ipq;
            const double rp = pk.p * ipq, rq = pb.p * ipq;
            if (lane == 0) boys_rt(P.boys, T, pb.K * pk.K * sq, F, lt);
            __syncwarp();
            // level 0: [e0|00]^(m), |e| <= lab, m <= lt - |e|, by |e|
            double* L0 = sm + G.lvl_off[0];
            for (int m = lane; m <= lt; m += 32) L0[m] = F[m];
            __syncwarp();
            for (int l = 1; l <= lab; l++) {
                const int nm = lt - l + 1, cnt = g_ncart(l) * nm;
                for (int t = lane; t < cnt; t += 32) {
                    const int idx = t / nm, m = t - idx * nm;
                    int e[3];
                    g_cart(l, idx, e[0], e[1], e[2]);
                    const int i = e[0] ? 0 : (e[1] ? 1 : 2);
                    int e1[3] = {e[0], e[1], e[2]};
                    e1[i]--;
                    const double* a = L0 + g_eoff(G, 0, l - 1, g_lidx(e1[0], e1[1], e1[2]));
                    double v = PA[i] * a[m] + WP[i] * a[m + 1];
                    if (e1[i] > 0) {
                        int e2[3] = {e1[0], e1[1], e1[2]};
                        e2[i]--;
                        const double* c = L0 + g_eoff(G, 0, l - 2, g_lidx(e2[0], e2[1], e2[2]));
                        v += e1[i] * o2p * (c[m] - rp * c[m + 1]);
                    }
                    L0[g_eoff(G, 0, l, idx) + m] = v;
                }
                __syncwarp();
            }
            // levels k = 1..lcd: [e0|f0]^(m) from levels k-1 and k-2
            for (int k = 0; k <= G.lcd; k++) {
                double* Lk = sm + G.lvl_off[k % 3];
                if (k > 0) {
                    const double* L1 = sm + G.lvl_off[(k + 2) % 3];   // level k-1
                    const double* L2 = sm + G.lvl_off[(k + 1) % 3];   // level k-2
                    const int fb1 = g_fblock(G, k - 1), fb0 = g_fblock(G, k);
                    const int fb2 = k >= 2 ? g_fblock(G, k - 2) : 0;
                    const int per_f = fb0;
                    const int cnt = g_ncart(k) * per_f;
                    for (int t = lane; t < cnt; t += 32) {
                        const int fidx = t / per_f;
                        int r = t - fidx * per_f;
                        // locate (e level l, e idx, m) inside the f block
                        int l = 0;
                        while (r >= g_ncart(l) * (lt - l - k + 1)) r -= g_ncart(l) * (lt - l - k + 1), l++;
                        const int nm = lt - l - k + 1;
                        const int eidx = r / nm, m = r - eidx * nm;
                        int e[3], f[3];
                        g_cart(l, eidx, e[0], e[1], e[2]);
                        g_cart(k, fidx, f[0], f[1], f[2]);
                        const int i = f[0] ? 0 : (f[1] ? 1 : 2);
                        int f1[3] = {f[0], f[1], f[2]};
                        f1[i]--;
                        const double* a = L1 + g_lidx(f1[0], f1[1], f1[2]) * fb1 + g_eoff(G, k - 1, l, eidx);
                        double v = QC[i] * a[m] + WQ[i] * a[m + 1];
                        if (f1[i] > 0) {
                            int f2[3] = {f1[0], f1[1], f1[2]};
                            f2[i]--;
                            const double* c = L2 + g_lidx(f2[0], f2[1], f2[2]) * fb2 + g_eoff(G, k - 2, l, eidx);
                            v += f1[i] * o2q * (c[m] - rq * c[m + 1]);
                        }
                        if (e[i] > 0) {
                            int e1[3] = {e[0], e[1], e[2]};
                            e1[i]--;
                            const double* c = L1 + g_lidx(f1[0], f1[1], f1[2]) * fb1 +
                                              g_eoff(G, k - 1, l - 1, g_lidx(e1[0], e1[1], e1[2]));
                            v += e[i] * o2pq * c[m + 1];
                        }
                        Lk[fidx * fb0 + g_eoff(G, k, l, eidx) + m] = v;
                    }
                    __syncwarp();
                }
                // contract the targets of this level
                if (k >= G.lc) {
                    const int fb0 = g_fblock(G, k);
                    const int nfl = g_ncart(k);
                    const int e0 = g_ncum(G.la - 1);
                    const int ntar = G.ne * nfl;
                    for (int t = lane; t < ntar; t += 32) {
                        const int ei = t / nfl, fidx = t - ei * nfl;
                        const int eg = e0 + ei;   // global e index
                        int l = 0;
                        while (g_ncum(l) <= eg) l++;
                        const int eidx = eg - g_ncum(l - 1);
                        const int fl = g_ncum(k - 1) - g_ncum(G.lc - 1) + fidx;
                        acc[ei * G.nf + fl] += Lk[fidx * fb0 + g_eoff(G, k, l, eidx)];
                    }
                }
                __syncwarp();
            }
        }
    }
    (void)lab;
}

// Digestion of the contracted block: closed-form horizontal recurrence per
// integral, six shared-memory accumulators, one flush per quartet.
__device__ void generic_digest(const QuartetCtx& q, const FockParams& P, const GenLayout& G, double* sm, int lane)
{
    const int la = G.la, lb = G.lb, lc = G.lc, ld = G.ld;
    const int na = g_ncart(la), nb = g_ncart(lb), nc = g_ncart(lc), nd = g_ncart(ld);
    const double* acc = sm + G.acc_off;
    double* Db = sm + G.d_off;
    double* Jb = sm + G.j_off;
    // density blocks: ab, cd, ac, ad, bc, bd
    const int o_ab = 0, o_cd = o_ab + na * nb, o_ac = o_cd + nc * nd, o_ad = o_ac + na * nc, o_bc = o_ad + na * nd,
              o_bd = o_bc + nb * nc, nblk = o_bd + nb * nd;
    const double* Dm = P.dense;
    const int n = P.nbasis;
    const int a0 = q.bfA, b0 = q.bfB, c0 = q.bfC, d0 = q.bfD;
    for (int t = lane; t < nblk; t += 32) {
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
    __syncwarp();
    const double AB[3] = {q.ABx, q.ABy, q.ABz}, CD[3] = {q.CDx, q.CDy, q.CDz};
    const bool exch = P.hybrid != 0.0;
    const int nout = na * nb * nc * nd;
    const int e0 = g_ncum(la - 1), f0 = g_ncum(lc - 1);
    for (int o = lane; o < nout; o += 32) {
        const int id = o % nd, ic = (o / nd) % nc, ib = (o / (nd * nc)) % nb, ia = o / (nd * nc * nb);
        const signed char* A = c_quick_cart[la][ia];
        const signed char* B = c_quick_cart[lb][ib];
        const signed char* Cc = c_quick_cart[lc][ic];
        const signed char* D = c_quick_cart[ld][id];
        double v = 0.0;
        for (int kx = 0; kx <= B[0]; kx++)
            for (int ky = 0; ky <= B[1]; ky++)
                for (int kz = 0; kz <= B[2]; kz++) {
                    const double cb = binom(B[0], kx) * binom(B[1], ky) * binom(B[2], kz) * ipow(AB[0], B[0] - kx) *
                                      ipow(AB[1], B[1] - ky) * ipow(AB[2], B[2] - kz);
                    const int ex = A[0] + kx, ey = A[1] + ky, ez = A[2] + kz;
                    const int eg = g_ncum(ex + ey + ez - 1) + g_lidx(ex, ey, ez) - e0;
                    double s = 0.0;
                    for (int jx = 0; jx <= D[0]; jx++)
                        for (int jy = 0; jy <= D[1]; jy++)
                            for (int jz = 0; jz <= D[2]; jz++) {
                                const double cd = binom(D[0], jx) * binom(D[1], jy) * binom(D[2], jz) *
                                                  ipow(CD[0], D[0] - jx) * ipow(CD[1], D[1] - jy) * ipow(CD[2], D[2] - jz);
                                const int fx = Cc[0] + jx, fy = Cc[1] + jy, fz = Cc[2] + jz;
                                const int fg = g_ncum(fx + fy + fz - 1) + g_lidx(fx, fy, fz) - f0;
                                s += cd * acc[eg * G.nf + fg];
                            }
                    v += cb * s;
                }
        atomicAdd(Jb + o_ab + ia * nb + ib, Db[o_cd + ic * nd + id] * v);
        atomicAdd(Jb + o_cd + ic * nd + id, Db[o_ab + ia * nb + ib] * v);
        if (exch) {
            atomicAdd(Jb + o_ac + ia * nc + ic, Db[o_bd + ib * nd + id] * v);
            atomicAdd(Jb + o_ad + ia * nd + id, Db[o_bc + ib * nc + ic] * v);
            atomicAdd(Jb + o_bc + ib * nc + ic, Db[o_ad + ia * nd + id] * v);
            atomicAdd(Jb + o_bd + ib * nd + id, Db[o_ac + ia * nc + ic] * v);
        }
    }
    __syncwarp();
    // flush with the weights of digest_coulomb / digest_exchange
    const double wj = 2.0 * q.w, wk = -0.5 * P.hybrid * q.w;
    for (int t = lane; t < (exch ? nblk : o_ac); t += 32) {
        int r, c;
        double wgt;
        if (t < o_cd) r = a0 + (t - o_ab) / nb, c = b0 + (t - o_ab) % nb, wgt = wj;
        else if (t < o_ac) r = c0 + (t - o_cd) / nd, c = d0 + (t - o_cd) % nd, wgt = wj;
        else if (t < o_ad) r = a0 + (t - o_ac) / nc, c = c0 + (t - o_ac) % nc, wgt = wk;
        else if (t < o_bc) r = a0 + (t - o_ad) / nd, c = d0 + (t - o_ad) % nd, wgt = wk;
        else if (t < o_bd) r = b0 + (t - o_bc) / nc, c = c0 + (t - o_bc) % nc, wgt = wk;
        else r = b0 + (t - o_bd) / nd, c = d0 + (t - o_bd) % nd, wgt = wk;
        fock_add(P.fock, n, r, c, wgt * Jb[t]);
    }
    __syncwarp();
}

// One warp (one block) per shell quartet; fp32_list: walk the class's FP32
// list (mixed precision) — these classes compute in FP64 either way.
__global__ void __launch_bounds__(32) fock_generic_kernel(const FockParams P, int cls, const GenLayout G, int fp32_list)
{
    extern __shared__ double sm[];
    const int lane = threadIdx.x;
    const int n = fp32_list ? P.class_count32[cls] : P.class_count[cls];
    const int2* list = fp32_list ? P.quartets + (P.class_end[cls] - n) : P.quartets + P.class_offset[cls];
    for (int i = blockIdx.x; i < n; i += gridDim.x) {
        QuartetCtx q;
        load_quartet(P, list[i], true, q);
        generic_quartet(q, P, G, sm, lane);
        generic_digest(q, P, G, sm, lane);
    }
}

int launch_generic_class(int cls, int la, int lb, int lc, int ld, const FockParams& P, int nq, int nsm, int fp32_list,
                         cudaStream_t st)
{
    if (nq <= 0) return 0;
    const GenLayout G = gen_layout(la, lb, lc, ld);
    const size_t bytes = (size_t)G.total * sizeof(double);
    int dev = 0, maxsm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxsm, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    if (bytes > (size_t)maxsm) return -1;
    static size_t configured = 0;
    if (bytes > 48 * 1024 && bytes > configured) {
        if (cudaFuncSetAttribute(fock_generic_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)maxsm) !=
            cudaSuccess)
            return -1;
        configured = maxsm;
    }
    int per_sm = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fock_generic_kernel, 32, bytes);
    const int grid = std::max(1, std::min(nq, nsm * std::max(per_sm, 1)));
    QB_LAUNCH(fock_generic_kernel, grid, 32, bytes, st, P, cls, G, fp32_list);
    return 32;
}

size_t generic_class_smem(int la, int lb, int lc, int ld)
{
    return (size_t)gen_layout(la, lb, lc, ld).total * sizeof(double);
}

}  // namespace qb
