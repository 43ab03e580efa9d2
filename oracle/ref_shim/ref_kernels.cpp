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

/* Shell-quartet counts of QUICK's own walk, kept per host thread and summed
   when the launch's threads finish:
     raw     every iclass call (ordered pair-pairs with ii <= kk that pass
             both Schwarz tests, gpu_get2e_subs.h:311-336);
     unique  the same walk counted once per unordered pair of pairs: for
             ii == kk only a <= b, and without the (p,s) copy of an sp
             shell's self-pair, whose integrals QUICK's basis-function
             filter drops (gpu_get2e_subs.h:792-801). */
static thread_local long long qref_raw_local = 0, qref_unique_local = 0;
static long long qref_raw = 0, qref_unique = 0;

static bool qref_sp_copy(int X, int Y)
{
    return devSim.sorted_Q[X] == devSim.sorted_Q[Y] && X != Y && devSim.sorted_Qnumber[X] > devSim.sorted_Qnumber[Y];
}

void qref_count_quartet(unsigned long long a, unsigned long long b, int II, int JJ, int KK, int LL, int ii, int kk)
{
    qref_raw_local++;
    if (qref_sp_copy(II, JJ) || qref_sp_copy(KK, LL)) return;
    if (ii < kk || a <= b) qref_unique_local++;
}

extern "C" void qref_quartet_counts(long long* raw, long long* unique)
{
    *raw = qref_raw;
    *unique = qref_unique;
}

extern "C" void qref_reset_counts(void) { qref_raw = qref_unique = 0; }

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
            __atomic_fetch_add(&qref_raw, qref_raw_local, __ATOMIC_RELAXED);
            __atomic_fetch_add(&qref_unique, qref_unique_local, __ATOMIC_RELAXED);
            qref_raw_local = qref_unique_local = 0;
        });
    }
    for (auto& th : pool) th.join();
}

/* QUICK's Boys function FmT (gpu_get2e_subs.h) at one argument, for checking
   its accuracy: out[m] = F_m(x) for m = 0..maxm. */
extern "C" void qref_fmt(int maxm, double x, double* out)
{
    QUICKDouble tmp[VDIM3];
    FmT(maxm, x, tmp);
    for (int m = 0; m <= maxm; m++) out[m] = tmp[m];
}

/* Boys function F_m(x) = int_0^1 t^(2m) exp(-x t^2) dt for m = 0..maxm,
   in long double: for x < 35 the series F_M = e^-x sum_k (2x)^k /
   ((2M+1)(2M+3)...(2M+2k+1)) for the top order and the stable downward
   recursion F_m = (2x F_(m+1) + e^-x) / (2m+1); above, F_0 =
   sqrt(pi/x) erf(sqrt x) / 2 and the (there stable) upward recursion. */
void qref_boys_accurate(int maxm, double xd, double* out)
{
    const long double x = xd;
    const long double e = expl(-x);
    if (x < 35.0L) {
        long double term = 1.0L / (2 * maxm + 1), sum = term;
        for (int k = 1; k < 2000; k++) {
            term *= 2.0L * x / (2 * maxm + 2 * k + 1);
            sum += term;
            if (term < 1e-22L * sum) break;
        }
        long double f = e * sum;
        out[maxm] = (double)f;
        for (int m = maxm - 1; m >= 0; m--) {
            f = (2.0L * x * f + e) / (2 * m + 1);
            out[m] = (double)f;
        }
    } else {
        long double f = 0.5L * sqrtl(3.14159265358979323846264338327950288L / x) * erfl(sqrtl(x));
        out[0] = (double)f;
        for (int m = 1; m <= maxm; m++) {
            f = ((2 * m - 1) * f - e) / (2.0L * x);
            out[m] = (double)f;
        }
    }
}
