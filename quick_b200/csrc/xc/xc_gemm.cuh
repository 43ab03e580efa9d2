// The dense steps of the XC quadrature on the FP64 tensor cores: a tiled
// C = A B with mma.sync m8n8k4 (FP64 in, FP64 accumulate), written for the
// three products of a grid chunk (xc.cu):
//   T0 = U phi   (U upper triangular: tiles left of the diagonal skipped)
//   S  = U^T psi (tiles right of the diagonal skipped)
//   M  = [phi' | chi'] [chi | phi]^T
// Operands are addressed by strides, one of which is 1 in each operand:
// element (m, k) of A at a[m * am + k * ak], (k, n) of B at b[k * bk + n * bn],
// (m, n) of C at c[m * cm + n * cn].
#pragma once
#include <cuda_runtime.h>

namespace qb {
namespace xcg {

constexpr int BM = 64, BN = 64, BK = 16;
constexpr int LDS = BM + 8;   // shared row stride (doubles): fragment loads hit each bank pair twice, the minimum

// Column j of tile row k sits at k * LDS + swz(j, k): the XOR of the low three
// bits with k spreads the tile stores of an operand whose unit stride is
// along K (16 consecutive k of one column per half-warp) over all banks
// instead of two (8-way conflicts before), and leaves the fragment loads
// and the other operand's stores at the two-wavefront minimum.
__device__ __forceinline__ int swz(int j, int k) { return j ^ (k & 7); }
constexpr int kThreads = 128; // 2 x 2 warps, 32 x 32 of C each

struct GemmArgs {
    const double* a;
    const double* b;
    double* c;
    long long am, ak, bk, bn, cm, cn;
    int M, N, K;
    int tri;        // 0: dense; 1: A upper triangular (A(m, k) = 0 for k < m); 2: A lower (0 for k > m)
    int kchunk;     // split K: slice z (blockIdx.z) sums k in [z kchunk, (z + 1) kchunk) into c + z cslice
    long long cslice;
};

// One tile row of an operand: rows r (the K index) x cols j (M or N index),
// 8 values per thread.  KFAST: the operand's unit stride is along K.
template <bool KFAST>
__device__ __forceinline__ void load_tile(const double* __restrict__ p, long long sj, long long sk, int j0, int k0,
                                          int J, int K, double* r)
{
    const int t = threadIdx.x;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        int j, k;
        if (KFAST) { k = t & 15; j = (t >> 4) + 8 * i; }
        else { j = t & 63; k = (t >> 6) + 2 * i; }
        const int gj = j0 + j, gk = k0 + k;
        r[i] = (gj < J && gk < K) ? __ldg(p + gj * sj + gk * sk) : 0.0;
    }
}

template <bool KFAST>
__device__ __forceinline__ void store_tile(double* s, const double* r)
{
    const int t = threadIdx.x;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        int j, k;
        if (KFAST) { k = t & 15; j = (t >> 4) + 8 * i; }
        else { j = t & 63; k = (t >> 6) + 2 * i; }
        s[k * LDS + swz(j, k)] = r[i];
    }
}

__device__ __forceinline__ void mma884(double& d0, double& d1, double a, double b)
{
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

template <bool AK, bool BK_>
__global__ void __launch_bounds__(kThreads) dmma_gemm_kernel(const GemmArgs g)
{
    __shared__ __align__(16) double As[2][BK * LDS];
    __shared__ __align__(16) double Bs[2][BK * LDS];
    // a slice can be empty for a triangular A: its partial C is still written (zeros)
    const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
    const int gid = lane >> 2, tig = lane & 3;
    int kb = blockIdx.z * g.kchunk, ke = min(g.K, kb + g.kchunk);
    if (g.tri == 1) kb = max(kb, (m0 / BK) * BK);
    if (g.tri == 2) ke = min(ke, m0 + BM);
    double* cz = g.c + blockIdx.z * g.cslice;
    double acc[4][4][2];
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) acc[i][j][0] = acc[i][j][1] = 0.0;
    double ra[8], rb[8];
    load_tile<AK>(g.a, g.am, g.ak, m0, kb, g.M, ke, ra);
    load_tile<BK_>(g.b, g.bn, g.bk, n0, kb, g.N, ke, rb);
    store_tile<AK>(As[0], ra);
    store_tile<BK_>(Bs[0], rb);
    __syncthreads();
    int buf = 0;
    for (int k0 = kb; k0 < ke; k0 += BK) {
        const bool more = k0 + BK < ke;
        if (more) {   // next tile into registers while this one is multiplied
            load_tile<AK>(g.a, g.am, g.ak, m0, k0 + BK, g.M, ke, ra);
            load_tile<BK_>(g.b, g.bn, g.bk, n0, k0 + BK, g.N, ke, rb);
        }
        const double* as = As[buf];
        const double* bs = Bs[buf];
#pragma unroll
        for (int kk = 0; kk < BK; kk += 4) {
            double fa[4], fb[4];
#pragma unroll
            for (int i = 0; i < 4; i++) fa[i] = as[(kk + tig) * LDS + swz(wm + 8 * i + gid, kk + tig)];
#pragma unroll
            for (int j = 0; j < 4; j++) fb[j] = bs[(kk + tig) * LDS + swz(wn + 8 * j + gid, kk + tig)];
#pragma unroll
            for (int i = 0; i < 4; i++)
#pragma unroll
                for (int j = 0; j < 4; j++) mma884(acc[i][j][0], acc[i][j][1], fa[i], fb[j]);
        }
        if (more) {
            store_tile<AK>(As[buf ^ 1], ra);
            store_tile<BK_>(Bs[buf ^ 1], rb);
        }
        __syncthreads();
        buf ^= 1;
    }
#pragma unroll
    for (int i = 0; i < 4; i++)
#pragma unroll
        for (int j = 0; j < 4; j++)
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int m = m0 + wm + 8 * i + gid, n = n0 + wn + 8 * j + 2 * tig + h;
                if (m < g.M && n < g.N) cz[m * g.cm + n * g.cn] = acc[i][j][h];
            }
}

// Launch C = A B on st; ak_unit / bk_unit: the operand's unit stride is along K.
// g.kchunk = 0: one slice over all of K.
inline void dmma_gemm(GemmArgs g, bool ak_unit, bool bk_unit, cudaStream_t st)
{
    if (g.kchunk <= 0) g.kchunk = g.K;
    dim3 grid((g.N + BN - 1) / BN, (g.M + BM - 1) / BM, (g.K + g.kchunk - 1) / g.kchunk);
    if (ak_unit && bk_unit) dmma_gemm_kernel<true, true><<<grid, kThreads, 0, st>>>(g);
    else if (ak_unit) dmma_gemm_kernel<true, false><<<grid, kThreads, 0, st>>>(g);
    else if (bk_unit) dmma_gemm_kernel<false, true><<<grid, kThreads, 0, st>>>(g);
    else dmma_gemm_kernel<false, false><<<grid, kThreads, 0, st>>>(g);
}

}  // namespace xcg
}  // namespace qb
