// One-electron integrals and their nuclear gradient on the GPU: the overlap
// S, the core Hamiltonian H = T + V and the one-electron part of the RHF
// gradient, over QUICK's angular sub-shells.  QUICK forms these on the host
// (fullx and get1eO/attrashell in src/quick_one_electron_integral.f90:18-126,
// 1633-1925, nuclearattra in src/nuclear.f90; hfgrad and attrashellopt in
// src/gradient.f90:49-249 and src/shell.f90:1747-1830); here one warp takes one
// pair of sub-shells:
//   * S and T from one-dimensional Obara-Saika overlap tables (the kinetic
//     operator as <d phi_a | d phi_b> / 2 per Cartesian direction), with
//     QUICK's per-function coefficients dcoeff;
//   * V by the Obara-Saika vertical recurrence [e|0]^(m) on the first centre
//     for every (primitive pair, nucleus) a lane takes, then the horizontal
//     transfer (a|b) = sum_k prod_i C(b_i,k_i) AB_i^(b_i-k_i) [a+k|0], with
//     QUICK's gccoeff x cons normalisation (nuclear.f90:198-221);
//   * the gradient from the same recurrences one order higher:
//     d/dA_i phi_a = 2 alpha phi_(a+1_i) - a_i phi_(a-1_i), the nucleus term
//     from translational invariance dV/dC = -(dV/dA + dV/dB), contracted on the
//     fly with D (and W for the overlap term).
// Lanes reduce with shuffles; the gradient accumulates per block in shared
// memory and is flushed once per block.
#include <algorithm>
#include <new>
#include <vector>
#include "eri_common.cuh"
#include "oneint.h"
#include "qb_internal.h"

namespace qb {

__host__ __device__ constexpr int nc_l(int l) { return (l + 1) * (l + 2) / 2; }
// Cartesian index inside shell n of (i, j, k), i+j+k = n: (n-i)(n-i+1)/2 + k
__device__ __forceinline__ int cart_in(int n, int i, int k) { return (n - i) * (n - i + 1) / 2 + k; }

// Vertical-recurrence table for total angular momentum <= LS: level n holds
// m = 0..LS-n, each a block of nc_l(n) entries.
template <int LS>
struct VrrTable {
    // sum over q < n of nc_l(q) (LS - q + 1), in closed form
    __host__ __device__ static constexpr int base(int n)
    {
        return (4 * (LS + 2) * n * (n + 1) * (n + 2) - 3 * n * n * (n + 1) * (n + 1) - 2 * n * (n + 1) * (2 * n + 1)) / 24;
    }
    static constexpr int size = base(LS + 1);
    static_assert(base(1) == LS + 1 && base(2) == 4 * LS + 1, "VrrTable::base");
    double v[size];
    __device__ __forceinline__ double& at(int n, int m, int c) { return v[base(n) + m * nc_l(n) + c]; }
};

// [e|0]^(m) for |e| <= LS from F_m (already scaled by the prefactor).
template <int LS>
__device__ __forceinline__ void vrr_attraction(VrrTable<LS>& T, const double* F, const double PA[3], const double PC[3],
                                               double o2p)
{
#pragma unroll
    for (int m = 0; m <= LS; m++) T.at(0, m, 0) = F[m];
#pragma unroll 1
    for (int n = 0; n < LS; n++) {
        const int n1 = n + 1;
        for (int i = n1; i >= 0; i--)
            for (int j = n1 - i; j >= 0; j--) {
                const int k = n1 - i - j;
                const int d = i > 0 ? 0 : (j > 0 ? 1 : 2);
                int e[3] = {i, j, k};
                e[d]--;
                const int nd = e[d];
                const int c1 = cart_in(n, e[0], e[2]);
                int c2 = 0;
                if (nd > 0) {
                    int f[3] = {e[0], e[1], e[2]};
                    f[d]--;
                    c2 = cart_in(n - 1, f[0], f[2]);
                }
                const int ct = cart_in(n1, i, k);
                for (int m = 0; m <= LS - n1; m++) {
                    double v = PA[d] * T.at(n, m, c1) - PC[d] * T.at(n, m + 1, c1);
                    if (nd > 0) v += nd * o2p * (T.at(n - 1, m, c2) - T.at(n - 1, m + 1, c2));
                    T.at(n1, m, ct) = v;
                }
            }
    }
}

// One-dimensional overlap table s[i][j], i <= NI, j <= NJ, without the
// prefactor (s[0][0] = 1).
template <int NI, int NJ>
__device__ __forceinline__ void overlap_1d(double (&s)[NI + 1][NJ + 1], double PA, double PB, double o2p)
{
    s[0][0] = 1.0;
#pragma unroll
    for (int i = 0; i < NI; i++) s[i + 1][0] = PA * s[i][0] + (i > 0 ? i * o2p * s[i - 1][0] : 0.0);
#pragma unroll
    for (int j = 0; j < NJ; j++)
#pragma unroll
        for (int i = 0; i <= NI; i++)
            s[i][j + 1] = PB * s[i][j] + o2p * ((i > 0 ? i * s[i - 1][j] : 0.0) + (j > 0 ? j * s[i][j - 1] : 0.0));
}

// kinetic 1-D element: (1/2)<d phi_i | d phi_j>
template <int NI, int NJ>
__device__ __forceinline__ double kinetic_1d(const double (&s)[NI + 1][NJ + 1], int i, int j, double a, double b)
{
    double t = 4.0 * a * b * s[i + 1][j + 1];
    if (i > 0) t -= 2.0 * b * i * s[i - 1][j + 1];
    if (j > 0) t -= 2.0 * a * j * s[i + 1][j - 1];
    if (i > 0 && j > 0) t += i * j * s[i - 1][j - 1];
    return 0.5 * t;
}

// Derivative along one direction of the 1-D overlap and kinetic factors with
// respect to the first centre: d/dA phi_i = 2a phi_(i+1) - i phi_(i-1).
template <int NI, int NJ>
__device__ __forceinline__ void deriv_1d(const double (&s)[NI + 1][NJ + 1], int i, int j, double a, double b,
                                         double& dS, double& dT)
{
    dS = 2.0 * a * s[i + 1][j];
    dT = 2.0 * a * kinetic_1d<NI, NJ>(s, i + 1, j, a, b);
    if (i > 0) {
        dS -= i * s[i - 1][j];
        dT -= i * kinetic_1d<NI, NJ>(s, i - 1, j, a, b);
    }
}

__host__ __device__ constexpr int ncum(int l) { return l < 0 ? 0 : (l + 1) * (l + 2) * (l + 3) / 6; }

// Adds w [e|0]^(0) for LMIN <= |e| <= LS to E (indexed from |e| = LMIN).
template <int LS, int LMIN>
__device__ __forceinline__ void add_level0(VrrTable<LS>& T, double w, double* E)
{
#pragma unroll 1
    for (int n = LMIN; n <= LS; n++) {
        const int b = ncum(n - 1) - ncum(LMIN - 1);
#pragma unroll 1
        for (int c = 0; c < nc_l(n); c++) E[b + c] += w * T.at(n, 0, c);
    }
}

// (a|b) = sum_k prod_i C(b_i,k_i) AB_i^(b_i-k_i) E[a+k], E indexed from |e| = LMIN.
template <int LMIN>
__device__ __forceinline__ double hrr_E(const double* E, int ax, int ay, int az, int bx, int by, int bz,
                                        const double AB[3])
{
    double s = 0.0;
    double cx = 1.0;
#pragma unroll 1
    for (int kx = bx; kx >= 0; kx--) {
        double cy = 1.0;
#pragma unroll 1
        for (int ky = by; ky >= 0; ky--) {
            double cz = 1.0;
#pragma unroll 1
            for (int kz = bz; kz >= 0; kz--) {
                const int ex = ax + kx, ez = az + kz, n = ex + ay + ky + ez;
                s += cx * cy * cz * E[ncum(n - 1) - ncum(LMIN - 1) + cart_in(n, ex, ez)];
                cz *= AB[2] * kz / (double)(bz - kz + 1);
            }
            cy *= AB[1] * ky / (double)(by - ky + 1);
        }
        cx *= AB[0] * kx / (double)(bx - kx + 1);
    }
    return s;
}

struct PairGeom {
    double A[3], B[3], AB[3], R2;
};

__device__ __forceinline__ PairGeom pair_geom(const OneIntParams& P, const OneQ& qa, const OneQ& qb)
{
    PairGeom g;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        g.A[d] = P.xyz[3 * qa.atom + d];
        g.B[d] = P.xyz[3 * qb.atom + d];
        g.AB[d] = g.A[d] - g.B[d];
    }
    g.R2 = g.AB[0] * g.AB[0] + g.AB[1] * g.AB[1] + g.AB[2] * g.AB[2];
    return g;
}

// [e|0]^(m) of one (primitive pair, nucleus) item, scaled by -Z_C and the
// contraction coefficients.  Returns false if the pair's overlap factor
// underflows.
template <int LS>
__device__ __forceinline__ bool attraction_item(const OneIntParams& P, const PairGeom& g, double a, double b,
                                                double cc, int C, VrrTable<LS>& T)
{
    const double p = a + b, ip = 1.0 / p;
    const double K = exp(-a * b * ip * g.R2);
    if (K < 1e-40) return false;
    double PA[3], PC[3];
    double PC2 = 0.0;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        const double Pd = (a * g.A[d] + b * g.B[d]) * ip;
        PA[d] = Pd - g.A[d];
        PC[d] = Pd - P.xyz[3 * C + d];
        PC2 += PC[d] * PC[d];
    }
    double F[LS + 1];
    boys<LS>(P.boys, p * PC2, 6.283185307179586477 * ip * K * -P.chg[C] * cc, F);
    vrr_attraction<LS>(T, F, PA, PC, 0.5 * ip);
    return true;
}

template <int LA, int LB>
__global__ void __launch_bounds__(128) oneint_kernel(const OneIntParams P, int begin, int end)
{
    constexpr int NA = nc_l(LA), NB = nc_l(LB), LS = LA + LB;
    constexpr int NE = ncum(LS) - ncum(LA - 1);
    constexpr int NMINE = (NA * NB + 31) / 32;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int w = begin + warp; w < end; w += nwarps) {
        const int2 pq = P.pairs[w];
        const OneQ qa = P.q[pq.x], qb = P.q[pq.y];
        const PairGeom g = pair_geom(P, qa, qb);
        double accS[NA * NB], accT[NA * NB], E[NE];
        for (int e = 0; e < NA * NB; e++) accS[e] = accT[e] = 0.0;
        for (int e = 0; e < NE; e++) E[e] = 0.0;
        const int npp = qa.np * qb.np;
        // overlap and kinetic energy, lanes over primitive pairs
        for (int t = lane; t < npp; t += 32) {
            const int ia = t / qb.np, ib = t - ia * qb.np;
            const double a = P.pexp[qa.poff + ia], b = P.pexp[qb.poff + ib], ip = 1.0 / (a + b);
            const double pref = 5.568327996831707845 * ip * sqrt(ip) * exp(-a * b * ip * g.R2);   // (pi/p)^(3/2) K
            double sx[LA + 2][LB + 2], sy[LA + 2][LB + 2], sz[LA + 2][LB + 2];
            const double o2p = 0.5 * ip;
            overlap_1d<LA + 1, LB + 1>(sx, -b * ip * g.AB[0], a * ip * g.AB[0], o2p);
            overlap_1d<LA + 1, LB + 1>(sy, -b * ip * g.AB[1], a * ip * g.AB[1], o2p);
            overlap_1d<LA + 1, LB + 1>(sz, -b * ip * g.AB[2], a * ip * g.AB[2], o2p);
#pragma unroll 1
            for (int mu = 0; mu < NA; mu++) {
                const int fa = qa.bf0 + mu;
                const int ix = P.itype[3 * fa], iy = P.itype[3 * fa + 1], iz = P.itype[3 * fa + 2];
                const double ca = P.dcoeff[(size_t)fa * P.maxcontract + ia] * pref;
#pragma unroll 1
                for (int nu = 0; nu < NB; nu++) {
                    const int fb = qb.bf0 + nu;
                    const int jx = P.itype[3 * fb], jy = P.itype[3 * fb + 1], jz = P.itype[3 * fb + 2];
                    const double c = ca * P.dcoeff[(size_t)fb * P.maxcontract + ib];
                    const double Sx = sx[ix][jx], Sy = sy[iy][jy], Sz = sz[iz][jz];
                    accS[mu * NB + nu] += c * Sx * Sy * Sz;
                    accT[mu * NB + nu] += c * (kinetic_1d<LA + 1, LB + 1>(sx, ix, jx, a, b) * Sy * Sz +
                                               Sx * kinetic_1d<LA + 1, LB + 1>(sy, iy, jy, a, b) * Sz +
                                               Sx * Sy * kinetic_1d<LA + 1, LB + 1>(sz, iz, jz, a, b));
                }
            }
        }
        // nuclear attraction: lanes over (primitive pair, nucleus) sum [e|0]
        // for LA <= |e| <= LA+LB; the transfer to (a|b) depends only on A-B
        for (int t = lane; t < npp * P.natom; t += 32) {
            const int pp = t / P.natom, C = t - pp * P.natom;
            const int ia = pp / qb.np, ib = pp - ia * qb.np;
            VrrTable<LS> T;
            if (attraction_item<LS>(P, g, P.pexp[qa.poff + ia], P.pexp[qb.poff + ib],
                                    P.pcoef[qa.poff + ia] * P.pcoef[qb.poff + ib], C, T))
                add_level0<LS, LA>(T, 1.0, E);
        }
#pragma unroll 1
        for (int e = 0; e < NE; e++) E[e] = warp_sum(E[e]);
        double mineS[NMINE], mineT[NMINE];
#pragma unroll 1
        for (int e = 0; e < NA * NB; e++) {
            const double s = warp_sum(accS[e]), t = warp_sum(accT[e]);
            if ((e & 31) == lane) {
                mineS[e >> 5] = s;
                mineT[e >> 5] = t;
            }
        }
        const bool diag = pq.x == pq.y;
#pragma unroll 1
        for (int e = lane; e < NA * NB; e += 32) {
            const int mu = e / NB, nu = e - mu * NB;
            if (diag && mu > nu) continue;
            const int fa = qa.bf0 + mu, fb = qb.bf0 + nu;
            const double v = hrr_E<LA>(E, P.klmn[3 * fa], P.klmn[3 * fa + 1], P.klmn[3 * fa + 2], P.klmn[3 * fb],
                                       P.klmn[3 * fb + 1], P.klmn[3 * fb + 2], g.AB);
            const double hv = mineT[e >> 5] + v * P.cons[fa] * P.cons[fb];
            const size_t i1 = fa + (size_t)fb * P.nbasis, i2 = fb + (size_t)fa * P.nbasis;
            if (P.S) P.S[i1] = P.S[i2] = mineS[e >> 5];
            if (P.H) P.H[i1] = P.H[i2] = hv;
        }
    }
}

template <int LA, int LB>
__global__ void __launch_bounds__(128) grad1e_kernel(const OneIntParams P, int begin, int end)
{
    constexpr int NA = nc_l(LA), NB = nc_l(LB), LS = LA + LB + 1;
    constexpr int LMIN = LA > 0 ? LA - 1 : 0;
    constexpr int NE = ncum(LS) - ncum(LMIN - 1);
    extern __shared__ double sg[];
    const bool shared_acc = P.grad_shared;
    if (shared_acc) {
        for (int i = threadIdx.x; i < 3 * P.natom; i += blockDim.x) sg[i] = 0.0;
        __syncthreads();
    }
    double* out = shared_acc ? sg : P.grad;
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    for (int w = begin + warp; w < end; w += nwarps) {
        const int2 pq = P.pairs[w];
        const OneQ qa = P.q[pq.x], qb = P.q[pq.y];
        const PairGeom g = pair_geom(P, qa, qb);
        // both orders of an off-diagonal block contribute
        const double fac = pq.x == pq.y ? 1.0 : 2.0;
        double gA[3] = {0, 0, 0}, gB[3] = {0, 0, 0};
        const int npp = qa.np * qb.np;
        // overlap (-W dS) and kinetic (D dT): two-centre, zero on one atom
        if (qa.atom != qb.atom) {
            for (int t = lane; t < npp; t += 32) {
                const int ia = t / qb.np, ib = t - ia * qb.np;
                const double a = P.pexp[qa.poff + ia], b = P.pexp[qb.poff + ib], ip = 1.0 / (a + b);
                const double pref = 5.568327996831707845 * ip * sqrt(ip) * exp(-a * b * ip * g.R2);
                double sx[LA + 3][LB + 2], sy[LA + 3][LB + 2], sz[LA + 3][LB + 2];
                const double o2p = 0.5 * ip;
                overlap_1d<LA + 2, LB + 1>(sx, -b * ip * g.AB[0], a * ip * g.AB[0], o2p);
                overlap_1d<LA + 2, LB + 1>(sy, -b * ip * g.AB[1], a * ip * g.AB[1], o2p);
                overlap_1d<LA + 2, LB + 1>(sz, -b * ip * g.AB[2], a * ip * g.AB[2], o2p);
#pragma unroll 1
                for (int mu = 0; mu < NA; mu++) {
                    const int fa = qa.bf0 + mu;
                    const int i3[3] = {P.itype[3 * fa], P.itype[3 * fa + 1], P.itype[3 * fa + 2]};
                    const double ca = P.dcoeff[(size_t)fa * P.maxcontract + ia] * pref * fac;
#pragma unroll 1
                    for (int nu = 0; nu < NB; nu++) {
                        const int fb = qb.bf0 + nu;
                        const int j3[3] = {P.itype[3 * fb], P.itype[3 * fb + 1], P.itype[3 * fb + 2]};
                        const double c = ca * P.dcoeff[(size_t)fb * P.maxcontract + ib];
                        const size_t ij = fa + (size_t)fb * P.nbasis;
                        const double dmu = P.D[ij], wmu = P.W[ij];
                        double S1[3], T1[3], dS[3], dT[3];
                        S1[0] = sx[i3[0]][j3[0]];
                        S1[1] = sy[i3[1]][j3[1]];
                        S1[2] = sz[i3[2]][j3[2]];
                        T1[0] = kinetic_1d<LA + 2, LB + 1>(sx, i3[0], j3[0], a, b);
                        T1[1] = kinetic_1d<LA + 2, LB + 1>(sy, i3[1], j3[1], a, b);
                        T1[2] = kinetic_1d<LA + 2, LB + 1>(sz, i3[2], j3[2], a, b);
                        deriv_1d<LA + 2, LB + 1>(sx, i3[0], j3[0], a, b, dS[0], dT[0]);
                        deriv_1d<LA + 2, LB + 1>(sy, i3[1], j3[1], a, b, dS[1], dT[1]);
                        deriv_1d<LA + 2, LB + 1>(sz, i3[2], j3[2], a, b, dS[2], dT[2]);
#pragma unroll
                        for (int d = 0; d < 3; d++) {
                            const int o1 = (d + 1) % 3, o2 = (d + 2) % 3;
                            // d/dA of S_x S_y S_z and of T = T_x S_y S_z + S_x T_y S_z + S_x S_y T_z
                            const double dSf = dS[d] * S1[o1] * S1[o2];
                            const double dTf = dT[d] * S1[o1] * S1[o2] + dS[d] * (T1[o1] * S1[o2] + S1[o1] * T1[o2]);
                            const double v = c * (dmu * dTf - wmu * dSf);
                            gA[d] += v;
                            gB[d] -= v;
                        }
                    }
                }
            }
        }
        // nuclear attraction: each lane takes whole nuclei, sums [e|0],
        // 2a [e|0] and 2b [e|0] over the primitive pairs, then contracts the
        // derivative integrals with D
        for (int C = lane; C < P.natom; C += 32) {
            if (C == qa.atom && C == qb.atom) continue;
            double E0[NE], E1[NE], E2[NE];
            for (int e = 0; e < NE; e++) E0[e] = E1[e] = E2[e] = 0.0;
#pragma unroll 1
            for (int pp = 0; pp < npp; pp++) {
                const int ia = pp / qb.np, ib = pp - ia * qb.np;
                const double a = P.pexp[qa.poff + ia], b = P.pexp[qb.poff + ib];
                VrrTable<LS> T;
                if (!attraction_item<LS>(P, g, a, b, P.pcoef[qa.poff + ia] * P.pcoef[qb.poff + ib], C, T)) continue;
                add_level0<LS, LMIN>(T, 1.0, E0);
                add_level0<LS, LMIN>(T, 2.0 * a, E1);
                add_level0<LS, LMIN>(T, 2.0 * b, E2);
            }
            double hA[3] = {0, 0, 0}, hB[3] = {0, 0, 0};
#pragma unroll 1
            for (int mu = 0; mu < NA; mu++) {
                const int fa = qa.bf0 + mu;
                const int ka[3] = {P.klmn[3 * fa], P.klmn[3 * fa + 1], P.klmn[3 * fa + 2]};
#pragma unroll 1
                for (int nu = 0; nu < NB; nu++) {
                    const int fb = qb.bf0 + nu;
                    const double wv = fac * P.D[fa + (size_t)fb * P.nbasis] * P.cons[fa] * P.cons[fb];
                    if (wv == 0.0) continue;
                    const int kb[3] = {P.klmn[3 * fb], P.klmn[3 * fb + 1], P.klmn[3 * fb + 2]};
#pragma unroll
                    for (int d = 0; d < 3; d++) {
                        int au[3] = {ka[0], ka[1], ka[2]}, bu[3] = {kb[0], kb[1], kb[2]};
                        au[d]++;
                        bu[d]++;
                        double dA = hrr_E<LMIN>(E1, au[0], au[1], au[2], kb[0], kb[1], kb[2], g.AB);
                        double dB = hrr_E<LMIN>(E2, ka[0], ka[1], ka[2], bu[0], bu[1], bu[2], g.AB);
                        if (ka[d] > 0) {
                            au[d] -= 2;
                            dA -= ka[d] * hrr_E<LMIN>(E0, au[0], au[1], au[2], kb[0], kb[1], kb[2], g.AB);
                        }
                        if (kb[d] > 0) {
                            bu[d] -= 2;
                            dB -= kb[d] * hrr_E<LMIN>(E0, ka[0], ka[1], ka[2], bu[0], bu[1], bu[2], g.AB);
                        }
                        hA[d] += wv * dA;
                        hB[d] += wv * dB;
                    }
                }
            }
#pragma unroll
            for (int d = 0; d < 3; d++) {
                gA[d] += hA[d];
                gB[d] += hB[d];
                atomicAdd(out + 3 * C + d, -(hA[d] + hB[d]));
            }
        }
#pragma unroll
        for (int d = 0; d < 3; d++) {
            const double xa = warp_sum(gA[d]), xb = warp_sum(gB[d]);
            if (lane == 0) {
                atomicAdd(out + 3 * qa.atom + d, xa);
                atomicAdd(out + 3 * qb.atom + d, xb);
            }
        }
    }
    if (shared_acc) {
        __syncthreads();
        for (int i = threadIdx.x; i < 3 * P.natom; i += blockDim.x)
            if (sg[i] != 0.0) atomicAdd(P.grad + i, sg[i]);
    }
}

// Nuclear repulsion gradient (hfgrad, src/gradient.f90:57-78), one thread per atom.
__global__ void nuclear_grad_kernel(const OneIntParams P)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= P.natom) return;
    double g[3] = {0, 0, 0};
    for (int j = 0; j < P.natom; j++) {
        if (j == i) continue;
        double d[3], r2 = 0.0;
        for (int k = 0; k < 3; k++) {
            d[k] = P.xyz[3 * j + k] - P.xyz[3 * i + k];
            r2 += d[k] * d[k];
        }
        const double f = P.chg[i] * P.chg[j] / (r2 * sqrt(r2));
        for (int k = 0; k < 3; k++) g[k] += d[k] * f;
    }
    for (int k = 0; k < 3; k++) P.grad[3 * i + k] += g[k];
}

template <int LA, int LB>
static void launch_pair_class(const OneIntParams& P, int begin, int end, int grad, int nsm, cudaStream_t st)
{
    const int n = end - begin;
    if (n <= 0) return;
    const int warps_per_block = 4;
    int grid = (n + warps_per_block - 1) / warps_per_block;
    grid = grid < nsm * 16 ? grid : nsm * 16;
    if (grad) {
        const size_t smem = P.grad_shared ? 3 * (size_t)P.natom * sizeof(double) : 0;
        grad1e_kernel<LA, LB><<<grid, 32 * warps_per_block, smem, st>>>(P, begin, end);
    } else {
        oneint_kernel<LA, LB><<<grid, 32 * warps_per_block, 0, st>>>(P, begin, end);
    }
}

#define QB_ONEINT_CASE(LA, LB) \
    case LA * 4 + LB: launch_pair_class<LA, LB>(P, begin, end, grad, nsm, st); return 0;

int launch_oneint_class(int la, int lb, const OneIntParams& P, int begin, int end, int grad, int nsm, cudaStream_t st)
{
    switch (la * 4 + lb) {
        QB_ONEINT_CASE(0, 0) QB_ONEINT_CASE(0, 1) QB_ONEINT_CASE(0, 2) QB_ONEINT_CASE(0, 3)
        QB_ONEINT_CASE(1, 0) QB_ONEINT_CASE(1, 1) QB_ONEINT_CASE(1, 2) QB_ONEINT_CASE(1, 3)
        QB_ONEINT_CASE(2, 0) QB_ONEINT_CASE(2, 1) QB_ONEINT_CASE(2, 2) QB_ONEINT_CASE(2, 3)
        QB_ONEINT_CASE(3, 0) QB_ONEINT_CASE(3, 1) QB_ONEINT_CASE(3, 2) QB_ONEINT_CASE(3, 3)
    default: return -1;
    }
}

void launch_nuclear_grad(const OneIntParams& P, cudaStream_t st)
{
    nuclear_grad_kernel<<<(P.natom + 127) / 128, 128, 0, st>>>(P);
}

// ------------------------------------------------------------------ host
namespace {

template <class T>
struct Buf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t put(const T* h, size_t count, cudaStream_t st)
    {
        if (count > n || !p) {
            if (p) cudaFree(p);
            p = nullptr;
            n = 0;
            cudaError_t e = cudaMalloc((void**)&p, std::max<size_t>(count, 1) * sizeof(T));
            if (e != cudaSuccess) return e;
            n = count;
        }
        return count ? cudaMemcpyAsync(p, h, count * sizeof(T), cudaMemcpyHostToDevice, st) : cudaSuccess;
    }
};

// Device copies of the sub-shell tables, rebuilt when the molecule changes.
struct OneIntTables {
    long long geom_version = -1;
    int device = -1;
    Buf<OneQ> q;
    Buf<int2> pairs;
    Buf<double> xyz, chg, aexp, dcoeff, cons, pexp, pcoef;
    Buf<int> itype, klmn;
    int cls_begin[16], cls_end[16];
    // host staging kept alive until the copies have run
    std::vector<OneQ> hq;
    std::vector<int2> hpairs;
    std::vector<double> hpexp, hpcoef;
};
OneIntTables g_tab;

int build_tables(const OneIntHost& h)
{
    int dev = -1;
    cudaGetDevice(&dev);
    if (g_tab.geom_version == h.geom_version && g_tab.device == dev) return 0;
    OneIntTables& t = g_tab;
    t.hq.clear();
    t.hpexp.clear();
    t.hpcoef.clear();
    for (int sh = 0; sh < h.nshell; sh++)
        for (int L = h.Qstart[sh]; L <= h.Qfinal[sh]; L++) {
            if (L > 3) return report_error(5, "one-electron integrals: angular momentum above f");
            OneQ q{};
            q.atom = h.katom[sh] - 1;
            q.L = L;
            q.bf0 = h.Ksumtype[sh] - 1 + h.Qsbasis[(size_t)sh + (size_t)L * h.nshell];
            q.np = h.kprim[sh];
            q.poff = (int)t.hpexp.size();
            for (int p = 0; p < q.np; p++) {
                t.hpexp.push_back(h.gcexpo[(size_t)p + (size_t)(h.Ksumtype[sh] - 1) * 10]);
                t.hpcoef.push_back(h.gccoeff[(size_t)p + (size_t)(h.Ksumtype[sh] - 1 + L) * 10]);
            }
            t.hq.push_back(q);
        }
    const int nq = (int)t.hq.size();
    std::vector<std::vector<int2>> by(16);
    for (int a = 0; a < nq; a++)
        for (int b = a; b < nq; b++) by[t.hq[a].L * 4 + t.hq[b].L].push_back(make_int2(a, b));
    t.hpairs.clear();
    for (int k = 0; k < 16; k++) {
        t.cls_begin[k] = (int)t.hpairs.size();
        t.hpairs.insert(t.hpairs.end(), by[k].begin(), by[k].end());
        t.cls_end[k] = (int)t.hpairs.size();
    }
    const size_t nb = h.nbasis, mc = h.maxcontract;
    cudaStream_t st = h.stream;
    cudaError_t e = cudaSuccess;
    if ((e = t.q.put(t.hq.data(), t.hq.size(), st)) != cudaSuccess ||
        (e = t.pairs.put(t.hpairs.data(), t.hpairs.size(), st)) != cudaSuccess ||
        (e = t.xyz.put(h.xyz, 3 * (size_t)h.natom, st)) != cudaSuccess ||
        (e = t.chg.put(h.chg, h.natom, st)) != cudaSuccess ||
        (e = t.aexp.put(h.aexp, mc * nb, st)) != cudaSuccess ||
        (e = t.dcoeff.put(h.dcoeff, mc * nb, st)) != cudaSuccess ||
        (e = t.cons.put(h.cons, nb, st)) != cudaSuccess ||
        (e = t.pexp.put(t.hpexp.data(), t.hpexp.size(), st)) != cudaSuccess ||
        (e = t.pcoef.put(t.hpcoef.data(), t.hpcoef.size(), st)) != cudaSuccess ||
        (e = t.itype.put(h.itype, 3 * nb, st)) != cudaSuccess ||
        (e = t.klmn.put(h.KLMN, 3 * nb, st)) != cudaSuccess)
        return report_error(2, cudaGetErrorString(e));
    // the staging vectors must outlive the asynchronous copies
    if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return report_error(2, cudaGetErrorString(e));
    t.geom_version = h.geom_version;
    t.device = dev;
    return 0;
}

OneIntParams params(const OneIntHost& h)
{
    OneIntParams P{};
    P.q = g_tab.q.p;
    P.pairs = g_tab.pairs.p;
    P.xyz = g_tab.xyz.p;
    P.chg = g_tab.chg.p;
    P.natom = h.natom;
    P.nbasis = h.nbasis;
    P.maxcontract = h.maxcontract;
    P.aexp = g_tab.aexp.p;
    P.dcoeff = g_tab.dcoeff.p;
    P.itype = g_tab.itype.p;
    P.klmn = g_tab.klmn.p;
    P.cons = g_tab.cons.p;
    P.pexp = g_tab.pexp.p;
    P.pcoef = g_tab.pcoef.p;
    P.boys = h.d_boys;
    return P;
}

}  // namespace

void oneint_release()
{
    OneIntTables& t = g_tab;
    void* ptrs[] = {t.q.p, t.pairs.p, t.xyz.p, t.chg.p, t.aexp.p, t.dcoeff.p, t.cons.p, t.pexp.p, t.pcoef.p,
                    t.itype.p, t.klmn.p};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    g_tab.~OneIntTables();
    new (&g_tab) OneIntTables();
}

int oneint_run(const OneIntHost& h, double* d_S, double* d_H)
{
    if (int rc = build_tables(h)) return rc;
    OneIntParams P = params(h);
    P.S = d_S;
    P.H = d_H;
    for (int k = 0; k < 16; k++)
        if (g_tab.cls_end[k] > g_tab.cls_begin[k]) {
            launch_oneint_class(k / 4, k % 4, P, g_tab.cls_begin[k], g_tab.cls_end[k], 0, h.nsm, h.stream);
            g_launches++;
        }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : report_error(2, cudaGetErrorString(e));
}

int grad1e_run(const OneIntHost& h, const double* d_D, const double* d_W, double* d_grad)
{
    if (int rc = build_tables(h)) return rc;
    OneIntParams P = params(h);
    P.D = d_D;
    P.W = d_W;
    P.grad = d_grad;
    P.grad_shared = 3 * (size_t)h.natom * sizeof(double) <= 48 * 1024;
    launch_nuclear_grad(P, h.stream);
    g_launches++;
    for (int k = 0; k < 16; k++)
        if (g_tab.cls_end[k] > g_tab.cls_begin[k]) {
            launch_oneint_class(k / 4, k % 4, P, g_tab.cls_begin[k], g_tab.cls_end[k], 1, h.nsm, h.stream);
            g_launches++;
        }
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? 0 : report_error(2, cudaGetErrorString(e));
}

}  // namespace qb
