/* Force-included shim that lets g++ compile QUICK's CUDA sources
 * (src/cuda/gpu.cu, gpu_get2e.cu) as plain host code.  This is test
 * infrastructure: it builds the checker, never the product.
 *
 *  - CUDA's own headers already turn __device__/__global__/__constant__ into
 *    nothing under a non-CUDA compiler; __launch_bounds__ is added here.
 *  - The launch geometry (blockIdx, blockDim, threadIdx, gridDim) is
 *    thread-local, so a "kernel" is run by N host threads, thread t playing
 *    block t of N one-thread blocks; QUICK's grid-stride loops then split
 *    their work across the threads.
 *  - atomicAdd on the 64-bit fixed-point accumulators becomes a relaxed GCC
 *    atomic, so the threads accumulate exactly as the GPU's atomics do.
 */
#pragma once
#include <cuda_runtime.h>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <cctype>
#include <cstdio>
using std::abs;

#ifndef __launch_bounds__
#define __launch_bounds__(...)
#endif

struct qref_dim { unsigned int x, y, z; };
extern thread_local qref_dim qref_blockIdx, qref_threadIdx, qref_blockDim, qref_gridDim;
#define blockIdx qref_blockIdx
#define threadIdx qref_threadIdx
#define blockDim qref_blockDim
#define gridDim qref_gridDim

static inline unsigned long long atomicAdd(unsigned long long* a, unsigned long long v)
{
    return __atomic_fetch_add(a, v, __ATOMIC_RELAXED);
}
static inline unsigned int atomicAdd(unsigned int* a, unsigned int v)
{
    return __atomic_fetch_add(a, v, __ATOMIC_RELAXED);
}

/* F_m(x), m = 0..maxm, to full double precision (ref_kernels.cpp); the
   accurate-Boys checker build calls it in place of QUICK's FmT. */
void qref_boys_accurate(int maxm, double x, double* out);

/* Counts one iclass call of QUICK's spd walk (gpu_get2e_subs.h:327-336):
   a and b index QUICK's pair list, II..LL its sorted Qshells, ii and kk the
   first shells of the two pairs (defined in ref_kernels.cpp; the call is
   added to a build-directory copy of gpu_get2e_subs.h by build_ref.py). */
void qref_count_quartet(unsigned long long a, unsigned long long b, int II, int JJ, int KK, int LL, int ii, int kk);

/* Runs the kernel named in a QUICK_SAFE_CALL launch expression on host
   threads (defined in ref_kernels.cpp). */
void qref_launch(const char* launch_expression);

/* cudaMemcpyToSymbol on a __constant__ object: on the host the symbol is an
   ordinary object, so the copy is a memcpy into it. */
template <class T>
static inline cudaError_t cudaMemcpyToSymbol(const T& symbol, const void* src, size_t count,
                                             size_t offset = 0,
                                             cudaMemcpyKind kind = cudaMemcpyHostToDevice)
{
    (void)kind;
    memcpy((char*)&symbol + offset, src, count);
    return cudaSuccess;
}
