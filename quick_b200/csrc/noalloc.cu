// qb_fock_device_static: the device-resident Fock build with all of its
// working memory taken from one fixed array compiled into this library, for
// callers that cannot allocate GPU memory while they run — for example a
// host program that hands the GPU's memory to its own pool allocator at
// start-up and forbids further cudaMalloc, or code that must not allocate
// between its set-up and its timed region.
//
// The working memory (per-class counters and offsets, the cons-scaled
// density, the Fock accumulator, the device programs of the f-shell classes
// that run the generic kernel, and the quartet lists) lives in
// g_fock_scratch below: kFockScratchBytes on every GPU that loads the
// library, held until the process exits.  Host code cannot use the array's
// name as a device address (on the host it names a stand-in), so the device
// address is fetched once per device with cudaGetSymbolAddress, with the
// session's device current, on the first call made on it.
//
// Every call shares the one array and it keeps the last call's contents;
// each call clears what must start at zero.  Calls that overlap on the GPU
// (other host threads, other streams) race on it and must not be made.
// Every quartet runs in FP64 here (the mixed split of qb_set_mixed_precision
// is not applied), and each call waits for its stream twice (for the class
// counts), so a call cannot be recorded into a CUDA graph.
#include <algorithm>
#include <cstdarg>
#include <cstdio>
#include <vector>

#include "../../include/quick_b200.h"
#include "gen/eri_classes.h"
#include "qb_internal.h"

namespace qb {

constexpr size_t kFockScratchBytes = (size_t)64 << 20;   // 64 MiB
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_fock_scratch[kFockScratchBytes];
static unsigned char* g_scratch_addr[kMaxDevices];

static size_t round256(size_t x) { return (x + 255) & ~(size_t)255; }

static int fail(int code, const char* fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    return report_error(code, buf);
}

#define CKS(call)                                                                              \
    do {                                                                                       \
        cudaError_t e_ = (call);                                                               \
        if (e_ != cudaSuccess) return fail(2, "%s failed: %s", #call, cudaGetErrorString(e_)); \
    } while (0)

}  // namespace qb

using namespace qb;

void qb::noalloc_reset()
{
    for (auto& p : g_scratch_addr) p = nullptr;
}

extern "C" int qb_fock_device_static(const double* d_dense, const double* d_o_in, double* d_o_out)
{
    SessionView v;
    if (int rc = session_view(&v)) return rc;
    int dev = 0;
    CKS(cudaGetDevice(&dev));
    if (dev != v.dev_id)
        return fail(1, "qb_fock_device_static: device %d is current but the session runs on device %d", dev, v.dev_id);
    if (dev < 0 || dev >= kMaxDevices) return fail(1, "qb_fock_device_static: device %d out of range", dev);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_fock_scratch);
        if (e != cudaSuccess || !p)
            return fail(2, "qb_fock_device_static: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
        g_scratch_addr[dev] = (unsigned char*)p;
    }
    unsigned char* base = g_scratch_addr[dev];
    const int n = v.P.nbasis;
    const int ncls = kNumClasses;
    // carve the fixed array
    size_t off = 0;
    auto take = [&](size_t bytes) { unsigned char* p = base + off; off += round256(bytes); return p; };
    auto* counts = (unsigned long long*)take(ncls * sizeof(unsigned long long));
    auto* counts32 = (unsigned long long*)take(ncls * sizeof(unsigned long long));
    auto* class_count = (int*)take(ncls * sizeof(int));
    auto* class_count32 = (int*)take(ncls * sizeof(int));
    auto* class_offset = (long long*)take(ncls * sizeof(long long));
    auto* overflow = (int*)take(sizeof(int));
    auto* d_cls = (ScreenClass*)take(ncls * sizeof(ScreenClass));
    auto* dense = (double*)take((size_t)n * n * sizeof(double));
    auto* fock = (double*)take((size_t)n * n * sizeof(double));
    if (off > kFockScratchBytes)
        return fail(4, "qb_fock_device_static: %d basis functions need %zu bytes of working memory before any "
                       "quartet; the fixed array holds %zu bytes (use qb_fock_device)", n, off, kFockScratchBytes);
    cudaStream_t st = v.stream;

    // Schwarz-only count per class: an upper bound for any density
    std::vector<ScreenClass> cls = v.cls;
    for (auto& c : cls) c.out_offset = 0, c.capacity = 0;
    CKS(cudaMemcpyAsync(d_cls, cls.data(), ncls * sizeof(ScreenClass), cudaMemcpyHostToDevice, st));
    CKS(cudaMemsetAsync(counts, 0, ncls * sizeof(unsigned long long), st));
    CKS(cudaMemsetAsync(counts32, 0, ncls * sizeof(unsigned long long), st));
    FockParams P = v.P;
    P.mixed_cut = 0.0;   // every quartet in FP64 here
    ScreenParams S{d_cls, counts, nullptr, counts32};
    launch_screen(S, P, ncls, 1, v.nsm, st);
    CKS(cudaGetLastError());
    std::vector<unsigned long long> cnt(ncls);
    CKS(cudaMemcpyAsync(cnt.data(), counts, ncls * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st));
    CKS(cudaStreamSynchronize(st));

    // the kernel each class runs, chosen as fock_build chooses it, and the
    // device programs of the classes that run the generic kernel
    std::vector<int> generic(ncls, 0);
    std::vector<unsigned char*> prog(ncls, nullptr);
    std::vector<size_t> prog_bytes(ncls, 0);
    for (int k = 0; k < ncls; k++) {
        const int* L = kClassL[k];
        generic[k] = kClassGeneric[k] || L[0] + L[1] + L[2] + L[3] >= v.generic_min_l;
        if (!generic[k] || cnt[k] == 0) continue;
        prog_bytes[k] = generic_program_bytes(L[0], L[1], L[2], L[3]);
        prog[k] = take(prog_bytes[k]);
    }
    if (off > kFockScratchBytes)
        return fail(4, "qb_fock_device_static: %d basis functions and the f-shell class programs need %zu bytes "
                       "before any quartet; the fixed array holds %zu bytes (use qb_fock_device)", n, off,
                    kFockScratchBytes);
    auto* quartets = (Quartet*)(base + off);
    const long long qcap = (long long)((kFockScratchBytes - off) / sizeof(Quartet));

    std::vector<long long> offs(ncls);
    long long total = 0;
    for (int k = 0; k < ncls; k++) {
        cls[k].out_offset = total;
        cls[k].capacity = (long long)cnt[k];
        offs[k] = total;
        total += (long long)cnt[k];
    }
    if (total > qcap)
        return fail(4, "qb_fock_device_static: this molecule screens to %lld shell quartets; the fixed array holds "
                       "%lld at %d basis functions (use qb_fock_device)", total, qcap, n);
    CKS(cudaMemcpyAsync(d_cls, cls.data(), ncls * sizeof(ScreenClass), cudaMemcpyHostToDevice, st));
    CKS(cudaMemcpyAsync(class_offset, offs.data(), ncls * sizeof(long long), cudaMemcpyHostToDevice, st));
    CKS(cudaMemsetAsync(counts, 0, ncls * sizeof(unsigned long long), st));
    CKS(cudaMemsetAsync(counts32, 0, ncls * sizeof(unsigned long long), st));
    CKS(cudaMemsetAsync(overflow, 0, sizeof(int), st));
    CKS(cudaMemsetAsync(fock, 0, (size_t)n * n * sizeof(double), st));

    // the Fock build proper, with the same kernels as qb_fock_device
    launch_scale_density(d_dense, v.cons, dense, n, st);
    P.quartets = quartets;
    P.class_offset = class_offset;
    P.class_count = class_count;
    P.class_count32 = class_count32;
    P.class_end = nullptr;   // read only by the FP32 class kernels, which are not launched here
    P.dense = dense;
    P.fock = fock;
    S.out = quartets;
    launch_screen(S, P, ncls, 0, v.nsm, st);
    launch_finish_counts(S, class_count, class_count32, overflow, ncls, st);
    CKS(cudaGetLastError());
    std::vector<int> ccount(ncls);
    int ovf = 0;
    CKS(cudaMemcpyAsync(ccount.data(), class_count, ncls * sizeof(int), cudaMemcpyDeviceToHost, st));
    CKS(cudaMemcpyAsync(&ovf, overflow, sizeof(int), cudaMemcpyDeviceToHost, st));
    CKS(cudaStreamSynchronize(st));
    if (ovf) return fail(3, "qb_fock_device_static: quartet list overflow (internal sizing error)");
    for (int k = 0; k < ncls; k++) {
        if (ccount[k] == 0) continue;
        const int* L = kClassL[k];
        const int rc = generic[k]
                           ? launch_generic_class_placed(k, L[0], L[1], L[2], L[3], P, ccount[k], v.nsm, prog[k],
                                                         prog_bytes[k], st)
                           : launch_class(k, P, v.group.empty() ? 1 : v.group[k], ccount[k], v.nsm, st);
        if (rc < 0)
            return fail(5, "qb_fock_device_static: class (%d%d|%d%d) could not be launched (%d)", L[0], L[1], L[2],
                        L[3], rc);
    }
    CKS(cudaGetLastError());
    launch_fock_finish(fock, v.cons, d_o_in, d_o_out, n, st, v.P.fixed_point);
    CKS(cudaGetLastError());
    CKS(cudaStreamSynchronize(st));
    return 0;
}
