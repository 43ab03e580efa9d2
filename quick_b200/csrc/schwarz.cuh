// Schwarz bounds on the GPU (QUICK computes them on the host:
// schwarz.f90:12-548).  One record per (shell pair, angular sub-shell pair);
// the generated schwarz_diag<LA,LB> evaluates the diagonal (ab|ab) block.
#pragma once
#include "eri_common.cuh"

namespace qb {

struct SchwarzParams {
    const double4* prim;       // primitive pairs, same layout as the Fock tables
    const int4* pair_bf;       // (first bf of A, first bf of B, prim offset, nprim)
    const double4* pair_AB;    // (A - B, unused)
    const double* cons;
    const double* boys;
    double* out_contracted;    // per record: max |(ab|ab)| cons^4, all primitives
    double* out_prim;          // per primitive pair: the same for that pair alone
};


template <int LA, int LB>
__device__ double schwarz_diag(const SchwarzParams& S, int rec, int p0, int np);

// mode 0: thread per record (contracted); mode 1: thread per primitive pair.
template <int LA, int LB>
__global__ void __launch_bounds__(128) schwarz_kernel(const SchwarzParams S, int begin, int end, int mode)
{
    const int stride = gridDim.x * blockDim.x;
    if (mode == 0) {
        for (int r = begin + blockIdx.x * blockDim.x + threadIdx.x; r < end; r += stride) {
            const int4 info = S.pair_bf[r];
            S.out_contracted[r] = schwarz_diag<LA, LB>(S, r, 0, info.w);
        }
    } else {
        // primitive pairs of records begin..end are contiguous in the table
        const int p_begin = S.pair_bf[begin].z;
        const int4 last = S.pair_bf[end - 1];
        const int p_end = last.z + last.w;
        for (int p = p_begin + blockIdx.x * blockDim.x + threadIdx.x; p < p_end; p += stride) {
            int lo = begin, hi = end - 1;     // record owning primitive pair p
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (S.pair_bf[mid].z <= p) lo = mid; else hi = mid - 1;
            }
            const int4 info = S.pair_bf[lo];
            S.out_prim[p] = schwarz_diag<LA, LB>(S, lo, p - info.z, 1);
        }
    }
}

int launch_schwarz(int type, const SchwarzParams& S, int begin, int end, int mode, int grid, int block, cudaStream_t st);
// The same for any pair type up to f with the generic recurrence program (eri_generic.cu).
int launch_generic_schwarz(int la, int lb, const SchwarzParams& S, int begin, int end, int mode, int nsm,
                           cudaStream_t st);

}  // namespace qb
