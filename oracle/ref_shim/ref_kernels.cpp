/* QUICK's two-electron kernels (src/cuda/gpu_get2e.cu and the headers it
   includes) compiled as host code for the oracle.  QUICK_SAFE_CALL is
   re-pointed at qref_launch so every kernel launch in gpu_get2e.cu runs the
   kernel body on host threads instead. */
#include "qref_shim.h"
#include "gpu.h"
#undef QUICK_SAFE_CALL
#define QUICK_SAFE_CALL(x) qref_launch(#x)
#include "gpu_get2e.cu"

#include <string>
#include <thread>
#include <vector>

thread_local qref_dim qref_blockIdx, qref_threadIdx, qref_blockDim, qref_gridDim;

static int qref_nthreads = 1;
static int qref_nvirtual = 0;   // 0: one virtual thread per host thread
extern "C" void qref_set_threads(int n) { qref_nthreads = n > 0 ? n : 1; }
/* Number of GPU threads the launch pretends to have (gridDim.x of one-thread
   blocks), run round-robin by the host threads.  getxc_kernel takes at most
   one point of each radial shell per thread, so it needs at least as many
   threads as the largest Lebedev sphere (194), as every real launch has. */
extern "C" void qref_set_virtual_threads(int n) { qref_nvirtual = n > 0 ? n : 0; }

typedef void (*qref_kernel_fn)();
static const struct { const char* name; qref_kernel_fn fn; } qref_kernels[] = {
    {"get2e_kernel", get2e_kernel},
    {"getGrad_kernel", getGrad_kernel},
    {"getGrad_kernel_spdf", getGrad_kernel_spdf},
    {"getGrad_kernel_spdf2", getGrad_kernel_spdf2},
    {"getxc_kernel", getxc_kernel},
#ifdef CUDA_SPDF
    {"get2e_kernel_spdf", get2e_kernel_spdf},
    {"get2e_kernel_spdf2", get2e_kernel_spdf2},
    {"get2e_kernel_spdf3", get2e_kernel_spdf3},
    {"get2e_kernel_spdf4", get2e_kernel_spdf4},
    {"get2e_kernel_spdf5", get2e_kernel_spdf5},
    {"get2e_kernel_spdf6", get2e_kernel_spdf6},
    {"get2e_kernel_spdf7", get2e_kernel_spdf7},
    {"get2e_kernel_spdf8", get2e_kernel_spdf8},
    {"get2e_kernel_spdf9", get2e_kernel_spdf9},
    {"get2e_kernel_spdf10", get2e_kernel_spdf10},
#endif
};

void qref_launch(const char* expr)
{
    std::string s(expr);
    size_t b = s.find_first_not_of("( ");
    size_t e = s.find("<<<");
    std::string name = s.substr(b, e - b);
    while (!name.empty() && name.back() == ' ') name.pop_back();
    qref_kernel_fn fn = nullptr;
    for (auto& k : qref_kernels)
        if (name == k.name) fn = k.fn;
    if (!fn) {
        fprintf(stderr, "qref_launch: kernel %s is not available in the host build\n", name.c_str());
        abort();
    }
    int n = qref_nthreads;
    int nv = qref_nvirtual > 0 ? qref_nvirtual : n;
    std::vector<std::thread> pool;
    for (int t = 0; t < n; t++) {
        pool.emplace_back([fn, t, n, nv]() {
            for (int v = t; v < nv; v += n) {
                qref_blockIdx = {(unsigned)v, 0, 0};
                qref_threadIdx = {0, 0, 0};
                qref_blockDim = {1, 1, 1};
                qref_gridDim = {(unsigned)nv, 1, 1};
                fn();
            }
        });
    }
    for (auto& th : pool) th.join();
}
