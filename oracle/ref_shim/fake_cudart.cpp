/* A host-memory stand-in for the few CUDA runtime calls QUICK's bridge
 * (src/cuda/gpu.cu, gpu_type.h) makes, so that the bridge's own host logic
 * (uploads, shell sorting, pair-list sort, fixed-point conversion) runs
 * unchanged on the CPU for the oracle.  "Device" memory is host memory;
 * copies are memcpy; one fake device is reported.  Signatures follow CUDA's
 * public runtime headers.  Test infrastructure only. */
#include <cuda_runtime.h>
#include <cstdlib>
#include <cstring>

extern "C" {

cudaError_t cudaMalloc(void** p, size_t n) { *p = calloc(n ? n : 1, 1); return *p ? cudaSuccess : cudaErrorMemoryAllocation; }
cudaError_t cudaFree(void* p) { free(p); return cudaSuccess; }
cudaError_t cudaHostAlloc(void** p, size_t n, unsigned int) { return cudaMalloc(p, n); }
cudaError_t cudaFreeHost(void* p) { free(p); return cudaSuccess; }
cudaError_t cudaHostGetDevicePointer(void** d, void* h, unsigned int) { *d = h; return cudaSuccess; }
cudaError_t cudaMemcpy(void* d, const void* s, size_t n, cudaMemcpyKind) { if (n) memmove(d, s, n); return cudaSuccess; }
cudaError_t cudaMemcpyAsync(void* d, const void* s, size_t n, cudaMemcpyKind, cudaStream_t) { if (n) memmove(d, s, n); return cudaSuccess; }
cudaError_t cudaStreamCreate(cudaStream_t* s) { *s = nullptr; return cudaSuccess; }
cudaError_t cudaStreamSynchronize(cudaStream_t) { return cudaSuccess; }
cudaError_t cudaGetDeviceCount(int* n) { *n = 1; return cudaSuccess; }
cudaError_t cudaGetDeviceProperties_v2(cudaDeviceProp* p, int)
{
    memset(p, 0, sizeof(*p));
    strcpy(p->name, "host (oracle)");
    p->major = 10; p->minor = 0;
    p->multiProcessorCount = 1;
    p->totalGlobalMem = (size_t)1 << 34;
    p->clockRate = 1000000;
    return cudaSuccess;
}
cudaError_t cudaSetDevice(int) { return cudaSuccess; }
cudaError_t cudaThreadSynchronize(void) { return cudaSuccess; }
cudaError_t cudaThreadExit(void) { return cudaSuccess; }
cudaError_t cudaDeviceSetCacheConfig(cudaFuncCache) { return cudaSuccess; }
cudaError_t cudaDeviceGetLimit(size_t* v, cudaLimit) { *v = 0; return cudaSuccess; }
cudaError_t cudaDeviceSetLimit(cudaLimit, size_t) { return cudaSuccess; }
const char* cudaGetErrorString(cudaError_t) { return "no error (host oracle)"; }

}
