// Quartet screening: builds, per angular-momentum class, the list of shell
// quartets that pass QUICK's Schwarz and density tests
// (gpu_get2e_subs.h:311-328), grouped by bra pair.  Replaces QUICK's dense
// walk over all sqrQshell^2 pair-pairs with a sorted, early-exit scan.
#include "eri_common.cuh"
#include "qb_internal.h"

namespace qb {

// One warp per (class, tile of kScreenTile consecutive bra pairs).  The kets
// of the class's ket type come in segments of equal primitive count, each
// sorted by Schwarz bound, descending, so the scan of a segment stops at the
// first chunk of kets whose bound product fails for every bra of the tile.
// For each chunk of 32 kets the warp tests all bras of the tile and writes
// their survivors as one contiguous run (bra by bra, kets ascending), so
// the quartets that share a chunk of ket pairs sit next to each other in the
// list: a class kernel block that walks a contiguous slice of the list
// reads each ket pair's primitive data from L1 once per tile instead of once
// per quartet.  count_only: Schwarz test only, just count (used once per
// geometry to size the lists).
constexpr int kScreenTile = 4;

__global__ void __launch_bounds__(256) screen_kernel(const ScreenParams S, const FockParams P, int count_only)
{
    const int cls = blockIdx.y;
    const ScreenClass c = S.cls[cls];
    const int lane = threadIdx.x & 31;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int nwarps = (gridDim.x * blockDim.x) >> 5;
    const double cut = P.integral_cutoff;
    const unsigned below = (1u << lane) - 1u;
    for (int a0 = c.bra_begin + warp * kScreenTile; a0 < c.bra_end; a0 += nwarps * kScreenTile) {
        const int nt = min(kScreenTile, c.bra_end - a0);
        double Ya[kScreenTile];
        int4 sa[kScreenTile];
        double Ymax = 0.0;
#pragma unroll
        for (int t = 0; t < kScreenTile; t++) {
            Ya[t] = t < nt ? P.pair_Y[a0 + t] : 0.0;
            sa[t] = t < nt ? P.pair_sh[a0 + t] : make_int4(0, 0, 0, 0);
            Ymax = fmax(Ymax, Ya[t]);
        }
        for (int sg = c.seg_begin; sg < c.seg_end; sg++) {
            const int2 seg = P.ket_segs[sg];
            if (c.same_type && seg.y <= a0) continue;   // every bra of the tile is >= a0
            const int kb = c.same_type ? max(a0, seg.x) : seg.x;
            for (int k0 = kb; k0 < seg.y; k0 += 32) {
                if (!(P.pair_Y[k0] * Ymax > cut)) break;      // sorted inside the segment: the rest fail too
                const int b = k0 + lane;
                const double Yb = b < seg.y ? P.pair_Y[b] : 0.0;
                int4 sb = make_int4(0, 0, 0, 0);
                if (!count_only && b < seg.y) sb = P.pair_sh[b];
                unsigned m[kScreenTile], m32[kScreenTile];
                double dnm[kScreenTile];
                int tot = 0, tot32 = 0;
#pragma unroll
                for (int t = 0; t < kScreenTile; t++) {
                    bool pass = false, low = false;
                    dnm[t] = 0.0;
                    // same pair type: kets b >= a only
                    if (t < nt && b < seg.y && (!c.same_type || b >= a0 + t)) {
                        const double yy = Yb * Ya[t];
                        if (yy > cut) {
                            if (count_only) {
                                pass = true;
                            } else {
                                dnm[t] = dn_max(P, sa[t].x, sa[t].y, sb.x, sb.y);
                                const double bound = yy * dnm[t];
                                pass = bound > cut;
                                low = pass && bound < P.mixed_cut;
                            }
                        }
                    }
                    m[t] = __ballot_sync(FULL, pass && !low);
                    m32[t] = __ballot_sync(FULL, low);
                    tot += __popc(m[t]);
                    tot32 += __popc(m32[t]);
                }
                if (tot + tot32 == 0) continue;
                unsigned long long base = 0, base32 = 0;
                if (lane == 0) {
                    if (tot) base = atomicAdd(S.counts + c.counter, (unsigned long long)tot);
                    if (tot32) base32 = atomicAdd(S.counts32 + c.counter, (unsigned long long)tot32);
                }
                if (count_only) continue;
                base = __shfl_sync(FULL, base, 0);
                base32 = __shfl_sync(FULL, base32, 0);
#pragma unroll
                for (int t = 0; t < kScreenTile; t++) {
                    if ((m[t] >> lane) & 1u) {
                        const unsigned long long pos = base + __popc(m[t] & below);
                        if (pos < (unsigned long long)c.capacity) S.out[c.out_offset + pos] = Quartet{a0 + t, b, dnm[t]};
                    } else if ((m32[t] >> lane) & 1u) {
                        const unsigned long long pos = base32 + __popc(m32[t] & below);
                        if (pos < (unsigned long long)c.capacity)
                            S.out[c.out_offset + c.capacity - 1 - pos] = Quartet{a0 + t, b, dnm[t]};
                    }
                    base += __popc(m[t]);
                    base32 += __popc(m32[t]);
                }
            }
        }
    }
}

// Clamp counters to capacities and publish them as int for the class
// kernels; the FP64 (front) and FP32 (back) lists share a class's region.
__global__ void finish_counts_kernel(const ScreenParams S, int* class_count, int* class_count32, int* overflow,
                                     int ncls)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < ncls) {
        unsigned long long n = S.counts[c], n32 = S.counts32[c];
        const unsigned long long cap = (unsigned long long)S.cls[c].capacity;
        if (n + n32 > cap) {
            atomicExch(overflow, 1);
            n = n > cap ? cap : n;
            n32 = n32 > cap - n ? cap - n : n32;
        }
        class_count[c] = (int)n;
        class_count32[c] = (int)n32;
    }
}

// QUICK scales every Cartesian component by cons() inside its horizontal
// recurrence (gpu_get2e_subs_hrr.h:42).  Here the scaling is folded into the
// density going in, D'(k,l) = cons(k) cons(l) D(k,l), and into the Fock
// matrix coming out, which costs nothing inside the class kernels.
__global__ void scale_density_kernel(const double* __restrict__ D, const double* __restrict__ cons,
                                     double* __restrict__ Ds, int n)
{
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < (size_t)n * n) {
        const int i = (int)(idx % n), j = (int)(idx / n);
        Ds[idx] = D[idx] * cons[i] * cons[j];
    }
}

// O_out(i,j) = O_in(i,j) + cons(i) cons(j) G(max(i,j), min(i,j)), column-major, symmetric;
// fixed: G holds 64-bit fixed point.
__global__ void fock_finish_kernel(const double* __restrict__ G, const double* __restrict__ cons,
                                   const double* __restrict__ Oin, double* __restrict__ Oout, int n, int fixed)
{
    const size_t idx = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < (size_t)n * n) {
        const int i = (int)(idx % n), j = (int)(idx / n);
        const int hi = i > j ? i : j, lo = i > j ? j : i;
        const size_t e = (size_t)hi * n + lo;
        const double g = fixed ? (double)reinterpret_cast<const long long*>(G)[e] / kFixedScale : G[e];
        Oout[idx] = Oin[idx] + cons[i] * cons[j] * g;
    }
}

void launch_screen(const ScreenParams& S, const FockParams& P, int ncls, int count_only, int nsm, cudaStream_t st,
                   int gx)
{
    dim3 grid(gx > 0 ? gx : nsm * 4, ncls);
    QB_LAUNCH(screen_kernel, grid, 256, 0, st, S, P, count_only);
}

void launch_finish_counts(const ScreenParams& S, int* class_count, int* class_count32, int* overflow, int ncls,
                          cudaStream_t st)
{
    QB_LAUNCH(finish_counts_kernel, (ncls + 63) / 64, 64, 0, st, S, class_count, class_count32, overflow, ncls);
}

// Class counts of one pass added to the build's totals.
__global__ void add_counts_kernel(const int* __restrict__ cnt, const int* __restrict__ cnt32, int* tot, int* tot32,
                                  int ncls)
{
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c < ncls) {
        tot[c] += cnt[c];
        tot32[c] += cnt32[c];
    }
}

void launch_add_counts(const int* cnt, const int* cnt32, int* tot, int* tot32, int ncls, cudaStream_t st)
{
    QB_LAUNCH(add_counts_kernel, (ncls + 63) / 64, 64, 0, st, cnt, cnt32, tot, tot32, ncls);
}

void launch_scale_density(const double* D, const double* cons, double* Ds, int n, cudaStream_t st)
{
    const size_t N = (size_t)n * n;
    QB_LAUNCH(scale_density_kernel, (unsigned)((N + 255) / 256), 256, 0, st, D, cons, Ds, n);
}

void launch_fock_finish(const double* G, const double* cons, const double* Oin, double* Oout, int n, cudaStream_t st,
                        int fixed)
{
    const size_t N = (size_t)n * n;
    QB_LAUNCH(fock_finish_kernel, (unsigned)((N + 255) / 256), 256, 0, st, G, cons, Oin, Oout, n, fixed);
}

// QUICK's density screen (densityCutoff / DNscreen, src/schwarz.f90:550-600)
// on the device: cut(I, J) = cut(J, I) = max |D| over the basis functions of
// shells I and J (shell I spans [first[I], first[I+1])).  One block per shell
// I, threads over the shells J >= I.
__global__ void density_screen_kernel(const double* __restrict__ D, const int* __restrict__ first, int nshell, int n,
                                      double* __restrict__ cut)
{
    const int I = blockIdx.x;
    const int i0 = first[I], i1 = first[I + 1];
    for (int J = I + threadIdx.x; J < nshell; J += blockDim.x) {
        const int j0 = first[J], j1 = first[J + 1];
        double m = 0.0;
        for (int j = j0; j < j1; j++)
            for (int i = i0; i < i1; i++) m = fmax(m, fabs(D[i + (size_t)j * n]));
        cut[I + (size_t)J * nshell] = m;
        cut[J + (size_t)I * nshell] = m;
    }
}

__global__ void add_vector_kernel(const double* __restrict__ x, double* __restrict__ y, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) y[i] += x[i];
}

void launch_density_screen(const double* D, const int* shell_first, int nshell, int n, double* cut, cudaStream_t st)
{
    QB_LAUNCH(density_screen_kernel, nshell, 128, 0, st, D, shell_first, nshell, n, cut);
}

void launch_add_vector(const double* x, double* y, int n, cudaStream_t st)
{
    QB_LAUNCH(add_vector_kernel, (n + 255) / 256, 256, 0, st, x, y, n);
}

}  // namespace qb
