// Measurement helpers exported through the C ABI: an FP64/FP32 FMA
// throughput probe (the roofline denominator for the FP64-pipe-bound ERI
// kernels; no vendor figure is used) and a counter of the primitive quartets
// the Fock build evaluates (the roofline numerator).
#include "eri_common.cuh"
#include "qb_internal.h"

namespace qb {

template <class T>
__global__ void __launch_bounds__(256) fma_probe_kernel(T* out, int iters, T seed)
{
    T a0 = seed + threadIdx.x, a1 = a0 + 1, a2 = a0 + 2, a3 = a0 + 3, a4 = a0 + 4, a5 = a0 + 5, a6 = a0 + 6, a7 = a0 + 7;
    const T m = (T)0.999999, c = (T)1e-7;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int k = 0; k < 16; k++) {
            a0 = a0 * m + c; a1 = a1 * m + c; a2 = a2 * m + c; a3 = a3 * m + c;
            a4 = a4 * m + c; a5 = a5 * m + c; a6 = a6 * m + c; a7 = a7 * m + c;
        }
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = a0 + a1 + a2 + a3 + a4 + a5 + a6 + a7;
}

// Per class: primitive quartets that pass the screen, for the quartet lists
// of the last Fock build.
__global__ void __launch_bounds__(256) count_prims_kernel(const FockParams P, int ncls, unsigned long long* out)
{
    const int cls = blockIdx.y;
    const int n = P.class_count[cls];
    const Quartet* list = P.quartets + P.class_offset[cls];
    unsigned long long mine = 0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        QuartetCtx q;
        load_quartet(P, list[i], true, q);
        for (int ib = 0; ib < q.nbra; ib++) {
            const double cpb = load_prim_aux(P.prim, q.bra_off + ib).z;
            for (int ik = 0; ik < q.nket; ik++)
                if (prim_survives(q, cpb, load_prim_aux(P.prim, q.ket_off + ik).z, P.prim_limit)) mine++;
        }
    }
    for (int o = 16; o > 0; o >>= 1) mine += __shfl_xor_sync(FULL, mine, o);
    if ((threadIdx.x & 31) == 0 && mine) atomicAdd(out + cls, mine);
}

int fma_probe(int fp64, int nsm, double* gflops, cudaStream_t st)
{
    const int block = 256, grid = nsm * 8, iters = 4096;
    void* buf = nullptr;
    if (cudaMalloc(&buf, (size_t)grid * block * 8) != cudaSuccess) return 2;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 5; rep++) {
        cudaEventRecord(e0, st);
        if (fp64) {
            auto k = fma_probe_kernel<double>;
            QB_LAUNCH(k, grid, block, 0, st, (double*)buf, iters, 1.0);
        } else {
            auto k = fma_probe_kernel<float>;
            QB_LAUNCH(k, grid, block, 0, st, (float*)buf, iters, 1.0f);
        }
        cudaEventRecord(e1, st);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0 && ms < best) best = ms;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    const double flops = 2.0 * 8 * 16 * (double)iters * grid * block;
    *gflops = flops / (best * 1e-3) / 1e9;
    return cudaGetLastError() == cudaSuccess ? 0 : 2;
}

void launch_count_prims(const FockParams& P, int ncls, unsigned long long* out, int nsm, cudaStream_t st)
{
    dim3 grid(nsm * 2, ncls);
    QB_LAUNCH(count_prims_kernel, grid, 256, 0, st, P, ncls, out);
}

}  // namespace qb
