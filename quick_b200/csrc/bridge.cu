// Host side of the C ABI: QUICK's gpu_* bridge (src/cuda/gpu.cu) rebuilt
// around device-resident, class-sorted shell-pair tables.
//
// Differences from QUICK's bridge, by design:
//  * device buffers are allocated once per geometry and reused every SCF
//    iteration (QUICK re-allocates o, dense and oULL per call);
//  * the Fock matrix accumulates in FP64 with device atomics after per-thread
//    and per-warp reduction, not as 64-bit fixed point with one atomic per
//    integral;
//  * quartets are screened into per-class work lists instead of testing all
//    sqrQshell^2 pair-pairs in every thread.
#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/quick_b200.h"
#include "gen/eri_classes.h"
#include "qb_internal.h"
#include "oneint.h"
#include "schwarz.cuh"
#include "grad_common.cuh"
#include "xc/xc_api.h"

namespace qb {

constexpr int MAXPRIM = 10;                                  // src/modules/quick_size_module.f90:37
constexpr double X0 = 5.9149671727956128778234784350536;    // sqrt(2 pi^2.5), gpu_common.h:196

template <class T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t count)
    {
        if (count <= n && p) return cudaSuccess;
        release();
        n = count;
        return cudaMalloc((void**)&p, std::max<size_t>(count, 1) * sizeof(T));
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// side streams for concurrent class launches (QB_CLASS_STREAMS = total streams, default 4)
constexpr int kSideStreams = 3;

struct Context {
    int dev_id = -1;
    bool inited = false;
    int nsm = 148;
    cudaStream_t own_stream = nullptr, stream = nullptr;
    // molecule
    int natom = 0, nbasis = 0, nelec = 0, imult = 1, molchg = 0, iAtomType = 0;
    int method = 0;
    std::vector<double> xyz;
    std::vector<int> iattype;
    std::vector<double> chg;
    // basis (QUICK arrays)
    int nshell = 0, nprim = 0, jshell = 0, jbasis = 0, maxcontract = 0;
    std::vector<int> kstart, katom, kprim, Ksumtype, Qnumber, Qstart, Qfinal, Qsbasis, Qfbasis, KLMN;
    std::vector<double> gccoeff, gcexpo, cons;
    std::vector<int> ncontract, itype, ncenter;     // per basis function (XC quadrature)
    std::vector<double> aexp, dcoeff;
    long long geom_version = 0;                     // bumped by every coordinate or basis upload
    bool have_basis = false;
    int Qshell = 0, maxL = 0;
    std::vector<int> sorted_Q, sorted_Qnumber;
    // QUICK's pair list
    std::vector<int> ref_xy;
    int fStart = 0, ffStart = 0;
    std::vector<double> YCutoff, cutPrim;
    bool have_pairs = false;
    // our pair table
    int npair = 0;
    std::vector<int> type_begin, type_end;
    // device tables
    DevBuf<double4> d_prim;
    DevBuf<PrimRec32> d_prim32;          // FP32 records of the same primitive pairs
    DevBuf<double4> d_pair_A;            // centre of each pair's first shell
    DevBuf<float> d_boys32;              // FP32 Boys records
    DevBuf<double> d_pair_Y, d_boys, d_dense, d_dense_raw, d_cons, d_fock, d_cut_matrix, d_o_in, d_o_out, d_grad;
    DevBuf<int> d_shell_atom;
    DevBuf<int4> d_pair_bf, d_pair_sh;
    DevBuf<double4> d_pair_AB;
    DevBuf<ScreenClass> d_screen_cls;
    DevBuf<unsigned long long> d_counts, d_counts32;
    DevBuf<int> d_class_count, d_class_count32, d_overflow;
    DevBuf<long long> d_class_offset, d_class_end;
    DevBuf<Quartet> d_quartets;
    DevBuf<int2> d_ket_segs;             // constant primitive-count segments of the pair table
    DevBuf<double> d_S1, d_H1, d_D1, d_W1, d_g1;   // host-pointer one-electron entry points
    DevBuf<int> d_shell_first;                      // Ksumtype - 1 (nshell + 1), for the device density screen
    long long shell_first_version = -1;
    std::vector<ScreenClass> screen_cls;
    // The quartet lists of one build are written in npass passes over
    // disjoint bra ranges when the whole list would pass the memory budget
    // (list_budget_bytes): pass p's classes are pass_cls[p * kNumClasses + k],
    // all passes sharing d_quartets.  npass = 1: one pass, the full ranges.
    int npass = 1;
    std::vector<ScreenClass> pass_cls;
    DevBuf<ScreenClass> d_pass_cls;
    DevBuf<long long> d_pass_offset, d_pass_end;
    DevBuf<int> d_total_count, d_total_count32;   // per class, summed over a build's passes
    std::vector<int> class_group;        // lanes per shell quartet of each class kernel
    std::vector<int> class_group32;      // the same for the FP32 class kernels of the mixed split
    std::vector<int> grad_group, grad_group32;   // lanes per quartet of the gradient kernels (empty: 1)
    HostTables host;                     // host copies of the pair and primitive tables (build_tables)
    bool tuned64 = false, tuned32 = false;   // set by qb_autotune_classes
    int generic_min_l = 99;              // classes with L sum >= this run the generic kernel (QB_GENERIC_MIN_L)
    // per-iteration
    // O (one-electron part) and the density as uploaded by
    // gpu_upload_calculated_, on the device; the host copy of O is made when
    // a host-side path (gpu_getxc_, gpu_addint_) first needs it
    DevBuf<double> d_o_up, d_dense_up;
    // gpu_schwarz_'s work arrays, kept between calls (grow only): a
    // cudaMalloc / cudaFree pair per call took from milliseconds to a second
    DevBuf<double4> sw_prim, sw_ab;
    DevBuf<int4> sw_bf;
    DevBuf<double> sw_oc, sw_op;
    std::vector<double> o_host;
    bool o_host_valid = false;
    bool have_calc = false;
    double integralCutoff = 1e-7, primLimit = 1e-7, DMCutoff = 1e-9, gradCutoff = 1e-7;
    std::vector<double> cutMatrix;
    bool have_cutoff = false;
    std::vector<double> grad_host;
    bool have_grad = false;
    double uploaded_energy = 0.0;        // gpu_upload_energy_ (no reader)
    // stats
    long long last_quartets = 0, last_quartets32 = 0;
    long long last_grad_quartets = 0;
    double last_ms_grad = 0.0;
    bool stats_pending = false;          // the last Fock build's counts are still on the device
    double mixed_cut = 0.0;      // Fock builds: quartets with Y Y DNMax below this run in FP32 (0: all FP64)
    int xc_grid = 1;             // grid of qb_xc_device: 1 SG1, 2 the 75 x 302 Becke grid
    int fixed_point = 0;         // Fock builds accumulate 64-bit fixed point (qb_set_fixed_point)
    double last_ms_xc_grad = 0.0;
    XcResult last_xc;
    double last_ms_eri = 0, last_ms_screen = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
    // side streams of the class launches (fock_build); nside < 0: not created yet
    int nside = -1;
    cudaStream_t side[kSideStreams] = {};
    cudaEvent_t side_ev[kSideStreams] = {};
    cudaEvent_t fork_ev = nullptr;
};

unsigned long long g_launches = 0;   // kernels launched by this library
AoIntOut* g_aoint_out = nullptr;      // descriptor of the current gpu_aoint_ slice (launch tables)
static long long g_geom_counter = 0; // process-wide, so a cached XC grid never outlives its molecule
static Context* g = nullptr;
static int g_status = 0;
static std::string g_err;

static void set_error(int code, const char* fmt, ...)
{
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (!g_status) {
        g_status = code;
        g_err = buf;
    }
    fprintf(stderr, "quick_b200: %s\n", buf);
}

#define CK(call)                                                                          \
    do {                                                                                  \
        cudaError_t e_ = (call);                                                          \
        if (e_ != cudaSuccess) {                                                          \
            set_error(2, "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
            return 2;                                                                     \
        }                                                                                 \
    } while (0)

static int require(bool cond, const char* what)
{
    if (!cond) {
        set_error(1, "%s", what);
        return 1;
    }
    return 0;
}

// ------------------------------------------------------------ Boys table
// F_m(k/32) for the device table, summed as a long-double series
// F_m(T) = e^-T sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1)) at the top m, then
// downward recursion, which is stable.
static void boys_table(std::vector<double>& tab)
{
    tab.assign(kBoysTableSize, 0.0);
    for (int k = 0; k < kBoysPoints; k++) {
        long double T = (long double)k / kBoysPerUnit;
        int mmax = kBoysExpCol - 1;
        long double term = 1.0L / (2 * mmax + 1), sum = term;
        for (int j = 1; j < 2000; j++) {
            term *= 2.0L * T / (2 * mmax + 2 * j + 1);
            sum += term;
            if (term < sum * 1e-22L) break;
        }
        long double e = expl(-T);
        long double f = e * sum;
        tab[(size_t)k * kBoysCols + kBoysExpCol] = (double)e;
        tab[(size_t)k * kBoysCols + mmax] = (double)f;
        for (int m = mmax - 1; m >= 0; m--) {
            f = (2.0L * T * f + e) / (2 * m + 1);
            tab[(size_t)k * kBoysCols + m] = (double)f;
        }
    }
    // per-order records (eri_common.cuh: kBoysLOff)
    for (int L = 0; L <= kBoysLMax; L++)
        for (int k = 0; k < kBoysPoints; k++) {
            double* r = tab.data() + kBoysLOff + ((size_t)L * kBoysPoints + k) * 8;
            for (int j = 0; j < 7; j++) r[j] = tab[(size_t)k * kBoysCols + L + j];
            r[7] = tab[(size_t)k * kBoysCols + kBoysExpCol];
        }
}

// FP32 records on the finer grid T_k = k/64: F_L, F_{L+1}, F_{L+2}, e^-T_k
// for L <= kBoysLMax, by the same series and downward recursion.
static void boys_table32(std::vector<float>& tab)
{
    tab.assign(kBoys32Size, 0.0f);
    const int mtop = kBoysLMax + 2;
    for (int k = 0; k < kBoys32Points; k++) {
        long double T = (long double)k / kBoys32PerUnit;
        long double term = 1.0L / (2 * mtop + 1), sum = term;
        for (int j = 1; j < 2000; j++) {
            term *= 2.0L * T / (2 * mtop + 2 * j + 1);
            sum += term;
            if (term < sum * 1e-22L) break;
        }
        long double e = expl(-T);
        std::vector<long double> F(mtop + 1);
        F[mtop] = e * sum;
        for (int m = mtop - 1; m >= 0; m--) F[m] = (2.0L * T * F[m + 1] + e) / (2 * m + 1);
        for (int L = 0; L <= kBoysLMax; L++) {
            float* r = tab.data() + ((size_t)L * kBoys32Points + k) * 4;
            r[0] = (float)F[L];
            r[1] = (float)F[L + 1];
            r[2] = (float)F[L + 2];
            r[3] = (float)e;
        }
    }
}

// ------------------------------------------------------------- pair list
// QUICK's shell-pair list (gpu.cu:401-1003, sort_method 0), restated with
// stable sorts.  QUICK bubble-sorts each (q,p) class with strict
// comparisons, which leaves equal keys in insertion order; a stable sort on
// the same key gives the identical sequence.
//   band 1: YCutoff > 1e-4, ordered by kprim(x)*kprim(y) descending, ties by
//           kprim(x) descending (gpu.cu:447-531);
//   band 2: 1e-10 < YCutoff <= 1e-4, ordered by YCutoff descending, then
//           stably by the same kprim key (gpu.cu:532-636).
// fStart / ffStart mark the first (d,f) and the first (p+q = 6) class.
static int build_pairlist(int Qshell, const int* sQ, const int* sQn, const int* kprim, int nshell,
                          const double* Y, std::vector<int>& xy, int& fStart, int& ffStart)
{
    xy.clear();
    fStart = 0;
    ffStart = 0;
    const double cut1 = 1e-10, cut2 = 1e-4;
    auto yv = [&](int x, int y) { return Y[(size_t)sQ[x] + (size_t)sQ[y] * nshell]; };
    auto kp = [&](int x) { return kprim[sQ[x]]; };
    for (int band = 0; band < 2; band++) {
        for (int qp = 0; qp <= 6; qp++)
            for (int q = 0; q <= 3; q++)
                for (int p = 0; p <= 3; p++) {
                    if (p + q != qp) continue;
                    std::vector<std::pair<int, int>> blk;
                    for (int i = 0; i < Qshell; i++)
                        for (int j = 0; j < Qshell; j++) {
                            if (sQn[i] != q || sQn[j] != p || sQ[i] > sQ[j]) continue;
                            double v = yv(i, j);
                            bool in = band == 0 ? (v > cut2) : (v <= cut2 && v > cut1);
                            if (in) blk.push_back({i, j});
                        }
                    if (band == 1)
                        std::stable_sort(blk.begin(), blk.end(), [&](const std::pair<int, int>& a, const std::pair<int, int>& b) {
                            return yv(a.first, a.second) > yv(b.first, b.second);
                        });
                    std::stable_sort(blk.begin(), blk.end(), [&](const std::pair<int, int>& a, const std::pair<int, int>& b) {
                        long pa = (long)kp(a.first) * kp(a.second), pb = (long)kp(b.first) * kp(b.second);
                        if (pa != pb) return pa > pb;
                        return kp(a.first) > kp(b.first);
                    });
                    int a_before = (int)xy.size() / 2;
                    for (auto& e : blk) {
                        xy.push_back(e.first);
                        xy.push_back(e.second);
                    }
                    if (!blk.empty()) {
                        if (q == 2 && p == 3 && (band == 0 || fStart == 0)) fStart = a_before;
                        if (p + q == 6 && (band == 0 || ffStart == 0)) ffStart = a_before;
                    }
                }
    }
    int a = (int)xy.size() / 2;
    if (ffStart == 0) ffStart = a;
    if (fStart == 0) fStart = a;
    return a;
}

// Shells sorted by angular momentum, stable in shell order (gpu.cu:1165-1218).
static void sort_qshells(Context& c)
{
    c.Qshell = 0;
    for (int i = 0; i < c.nshell; i++) c.Qshell += c.Qfinal[i] - c.Qstart[i] + 1;
    c.sorted_Q.clear();
    c.sorted_Qnumber.clear();
    for (int L = 0; L <= 3; L++)
        for (int s = 0; s < c.nshell; s++)
            if (c.Qstart[s] <= L && L <= c.Qfinal[s]) {
                c.sorted_Q.push_back(s);
                c.sorted_Qnumber.push_back(L);
            }
    c.maxL = 0;
    for (int v : c.sorted_Qnumber) c.maxL = std::max(c.maxL, v);
}

static inline double ccoef(const Context& c, int sh, int L, int p)
{
    return c.gccoeff[(size_t)p + (size_t)(c.Ksumtype[sh] - 1 + L) * MAXPRIM];
}
static inline double cexpo(const Context& c, int sh, int p)
{
    return c.gcexpo[(size_t)p + (size_t)(c.Ksumtype[sh] - 1) * MAXPRIM];
}
static inline int bf_first(const Context& c, int sh, int L)
{
    return c.Ksumtype[sh] - 1 + c.Qsbasis[(size_t)sh + (size_t)L * c.nshell];
}
static inline const double* center(const Context& c, int sh) { return c.xyz.data() + 3 * (c.katom[sh] - 1); }

static int pair_type_index(int la, int lb)
{
    for (int t = 0; t < kNumPairTypes; t++)
        if (kPairTypeL[t][0] == la && kPairTypeL[t][1] == lb) return t;
    return -1;
}

// Our pair table from QUICK's list: drop the (p,s) copies of an sp shell's
// self-pair (QUICK lists both (s,p) and (p,s); its basis-function filter
// discards every integral of the second), orient each pair with the higher
// angular momentum first, group by pair type and sort by Schwarz bound.
static int build_tables(Context& c)
{
    struct Rec {
        int type, shA, shB, LA, LB, ref, key, np;
        double Y, w;
    };
    std::vector<Rec> recs;
    int npref = (int)c.ref_xy.size() / 2;
    for (int r = 0; r < npref; r++) {
        int x = c.ref_xy[2 * r], y = c.ref_xy[2 * r + 1];
        int sx = c.sorted_Q[x], sy = c.sorted_Q[y], Lx = c.sorted_Qnumber[x], Ly = c.sorted_Qnumber[y];
        if (sx == sy && x != y && Lx > Ly) continue;
        Rec e;
        e.ref = r;
        e.Y = c.YCutoff[(size_t)sx + (size_t)sy * c.nshell];
        e.w = (x == y) ? 0.5 : 1.0;
        e.key = sx * 4 + Lx;
        if (Lx >= Ly) { e.shA = sx; e.LA = Lx; e.shB = sy; e.LB = Ly; }
        else { e.shA = sy; e.LA = Ly; e.shB = sx; e.LB = Lx; }
        e.type = pair_type_index(e.LA, e.LB);
        if (e.type < 0) return set_error(1, "angular momentum (%d,%d) beyond this build", e.LA, e.LB), 1;
        e.np = c.kprim[e.shA] * c.kprim[e.shB];
        recs.push_back(e);
    }
    // by pair type, then primitive-pair count (descending), then Schwarz
    // bound (descending): the screen walks each constant-count segment in
    // bound order, so the quartets of one bra come out grouped by the ket's
    // primitive count and the lanes of a warp run loops of equal length
    std::stable_sort(recs.begin(), recs.end(), [](const Rec& a, const Rec& b) {
        if (a.type != b.type) return a.type < b.type;
        if (a.np != b.np) return a.np > b.np;
        return a.Y > b.Y;
    });
    c.npair = (int)recs.size();
    c.type_begin.assign(kNumPairTypes, 0);
    c.type_end.assign(kNumPairTypes, 0);
    for (int t = 0, i = 0; t < kNumPairTypes; t++) {
        c.type_begin[t] = i;
        while (i < c.npair && recs[i].type == t) i++;
        c.type_end[t] = i;
    }
    // constant primitive-count segments of each pair type
    std::vector<int2> segs;
    std::vector<int> tseg_begin(kNumPairTypes), tseg_end(kNumPairTypes);
    for (int t = 0; t < kNumPairTypes; t++) {
        tseg_begin[t] = (int)segs.size();
        for (int i = c.type_begin[t]; i < c.type_end[t];) {
            int j = i;
            while (j < c.type_end[t] && recs[j].np == recs[i].np) j++;
            segs.push_back(make_int2(i, j));
            i = j;
        }
        tseg_end[t] = (int)segs.size();
    }
    CK(c.d_ket_segs.alloc(std::max<size_t>(segs.size(), 1)));
    if (!segs.empty())
        CK(cudaMemcpy(c.d_ket_segs.p, segs.data(), segs.size() * sizeof(int2), cudaMemcpyHostToDevice));
    std::vector<int4> pbf(c.npair), psh(c.npair);
    std::vector<double> pY(c.npair);
    std::vector<double4> pAB(c.npair);
    std::vector<double4> prim;
    std::vector<PrimRec32> prim32;
    std::vector<double4> pA(c.npair);
    for (int i = 0; i < c.npair; i++) {
        const Rec& e = recs[i];
        const double *A = center(c, e.shA), *B = center(c, e.shB);
        double AB2 = 0;
        for (int k = 0; k < 3; k++) AB2 += (A[k] - B[k]) * (A[k] - B[k]);
        int off = (int)prim.size() / 3;
        // QUICK's own orientation (first Qshell x) indexes cutPrim
        int x = c.ref_xy[2 * e.ref], y = c.ref_xy[2 * e.ref + 1];
        int sx = c.sorted_Q[x], sy = c.sorted_Q[y];
        for (int pa = 0; pa < c.kprim[e.shA]; pa++)
            for (int pb = 0; pb < c.kprim[e.shB]; pb++) {
                double a = cexpo(c, e.shA, pa), b = cexpo(c, e.shB, pb), p = a + b;
                double X = exp(-a * b / p * AB2) / p;
                double K = X0 * X * ccoef(c, e.shA, e.LA, pa) * ccoef(c, e.shB, e.LB, pb);
                double P[3], PA[3];
                for (int k = 0; k < 3; k++) {
                    P[k] = (A[k] * a + B[k] * b) / p;
                    PA[k] = P[k] - A[k];
                }
                int px = (e.shA == sx && (sx != sy || e.LA == c.sorted_Qnumber[x])) ? pa : pb;
                int py = (px == pa) ? pb : pa;
                double cp = c.cutPrim[(size_t)(c.kstart[sx] - 1 + px) + (size_t)(c.kstart[sy] - 1 + py) * c.jbasis];
                prim.push_back(make_double4(p, K, P[0], P[1]));
                prim.push_back(make_double4(P[2], PA[0], PA[1], PA[2]));
                prim.push_back(make_double4(0.5 / p, a, cp, 0.0));
                PrimRec32 r32;
                r32.p = (float)p; r32.K = (float)K;
                r32.PAx = (float)PA[0]; r32.PAy = (float)PA[1]; r32.PAz = (float)PA[2];
                r32.alpha = (float)a;
                r32.cp = cp;
                prim32.push_back(r32);
            }
        pbf[i] = make_int4(bf_first(c, e.shA, e.LA), bf_first(c, e.shB, e.LB), off, (int)prim.size() / 3 - off);
        psh[i] = make_int4(e.shA, e.shB, e.key, e.ref);
        pY[i] = e.Y;
        pAB[i] = make_double4(A[0] - B[0], A[1] - B[1], A[2] - B[2], e.w);
        pA[i] = make_double4(A[0], A[1], A[2], 0.0);
    }
    CK(c.d_prim.alloc(prim.size()));
    CK(c.d_pair_bf.alloc(c.npair));
    CK(c.d_pair_sh.alloc(c.npair));
    CK(c.d_pair_Y.alloc(c.npair));
    CK(c.d_pair_AB.alloc(c.npair));
    CK(cudaMemcpy(c.d_prim.p, prim.data(), prim.size() * sizeof(double4), cudaMemcpyHostToDevice));
    CK(c.d_prim32.alloc(std::max<size_t>(prim32.size(), 1)));
    CK(c.d_pair_A.alloc(std::max<size_t>(pA.size(), 1)));
    if (!prim32.empty())
        CK(cudaMemcpy(c.d_prim32.p, prim32.data(), prim32.size() * sizeof(PrimRec32), cudaMemcpyHostToDevice));
    if (!pA.empty()) CK(cudaMemcpy(c.d_pair_A.p, pA.data(), pA.size() * sizeof(double4), cudaMemcpyHostToDevice));
    std::vector<int> satom(c.nshell);
    for (int s = 0; s < c.nshell; s++) satom[s] = c.katom[s] - 1;
    CK(c.d_shell_atom.alloc(c.nshell));
    CK(cudaMemcpy(c.d_shell_atom.p, satom.data(), c.nshell * sizeof(int), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.d_pair_bf.p, pbf.data(), pbf.size() * sizeof(int4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.d_pair_sh.p, psh.data(), psh.size() * sizeof(int4), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.d_pair_Y.p, pY.data(), pY.size() * sizeof(double), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.d_pair_AB.p, pAB.data(), pAB.size() * sizeof(double4), cudaMemcpyHostToDevice));
    // screening classes
    c.screen_cls.assign(kNumClasses, ScreenClass{});
    for (int k = 0; k < kNumClasses; k++) {
        int tb = pair_type_index(kClassL[k][0], kClassL[k][1]);
        int tk = pair_type_index(kClassL[k][2], kClassL[k][3]);
        ScreenClass& s = c.screen_cls[k];
        s.bra_begin = c.type_begin[tb];
        s.bra_end = c.type_end[tb];
        s.ket_begin = c.type_begin[tk];
        s.ket_end = c.type_end[tk];
        s.seg_begin = tseg_begin[tk];
        s.seg_end = tseg_end[tk];
        s.same_type = tb == tk;
        s.counter = k;
        s.out_offset = 0;
        s.capacity = 0;
    }
    // host copies of the molecule's tables, for a many-molecule batch (batch.cu)
    HostTables& h = c.host;
    h.nbasis = c.nbasis;
    h.nshell = c.nshell;
    h.natom = c.natom;
    h.pbf = pbf;
    h.psh = psh;
    h.pY = pY;
    h.pAB = pAB;
    h.pA = pA;
    h.prim = prim;
    h.prim32 = prim32;
    h.segs = segs;
    h.scls = c.screen_cls;
    h.cons = c.cons;
    h.shell_atom = satom;
    h.shell_first.resize(c.nshell + 1);
    for (int sh = 0; sh <= c.nshell; sh++) h.shell_first[sh] = c.Ksumtype[sh] - 1;
    // lanes per shell quartet: the class's mean primitive quartets before
    // screening (mean primitive pairs of the bra type x of the ket type) over
    // QB_FOCK_GDIV (default 2), rounded down to a power of two and clamped to
    // what the class was compiled for; QB_FOCK_G forces one value
    std::vector<double> type_prims(kNumPairTypes, 0.0);
    for (int t = 0; t < kNumPairTypes; t++) {
        double sum = 0.0;
        for (int i = c.type_begin[t]; i < c.type_end[t]; i++) sum += pbf[i].w;
        type_prims[t] = c.type_end[t] > c.type_begin[t] ? sum / (c.type_end[t] - c.type_begin[t]) : 0.0;
    }
    const char* gd = getenv("QB_FOCK_GDIV");
    const char* gf = getenv("QB_FOCK_G");
    const double div = gd && atof(gd) > 0 ? atof(gd) : 2.0;
    const char* gm = getenv("QB_GENERIC_MIN_L");
    c.generic_min_l = gm && atoi(gm) > 0 ? atoi(gm) : 99;
    // lane groups chosen by qb_autotune_classes stay for the following
    // molecules of the session
    if (c.tuned64 && c.tuned32) return 0;
    std::vector<int> keep64 = c.class_group, keep32 = c.class_group32;
    c.class_group.assign(kNumClasses, 1);
    for (int k = 0; k < kNumClasses; k++) {
        double est = type_prims[pair_type_index(kClassL[k][0], kClassL[k][1])] *
                     type_prims[pair_type_index(kClassL[k][2], kClassL[k][3])] / div;
        // at most 2 lanes before tuning: qb_autotune_classes on
        // (H2O)32/6-31G** picks 1 or 2 lanes for every class (4 for two FP32
        // light classes), and 8 lanes ran psss 1.8x slower than 2
        int g = 1;
        while (g * 2 <= est && g < 2) g *= 2;
        if (gf && atoi(gf) > 0) g = atoi(gf);   // QB_FOCK_G forces one value
        c.class_group[k] = std::min(g, class_max_group(k));
    }
    c.class_group32 = c.class_group;
    if (c.tuned64) c.class_group = keep64;
    if (c.tuned32) c.class_group32 = keep32;
    return 0;
}

static FockParams fock_params(Context& c)
{
    FockParams P;
    P.prim = c.d_prim.p;
    P.pair_bf = c.d_pair_bf.p;
    P.pair_sh = c.d_pair_sh.p;
    P.pair_Y = c.d_pair_Y.p;
    P.pair_AB = c.d_pair_AB.p;
    P.quartets = c.d_quartets.p;
    // the lists in the buffer: the last pass's (the only one unless the
    // lists were cut into passes)
    const size_t last = (size_t)(c.npass - 1) * kNumClasses;
    P.class_offset = c.d_pass_offset.p ? c.d_pass_offset.p + last : c.d_class_offset.p;
    P.class_count = c.d_class_count.p;
    P.dense = c.d_dense.p;
    P.fock = c.d_fock.p;
    P.cut_matrix = c.d_cut_matrix.p;
    P.boys = c.d_boys.p;
    P.nbasis = c.nbasis;
    P.nshell = c.nshell;
    P.prim_limit = c.primLimit;
    P.hybrid = c.method == 0 ? 1.0 : (c.method == 1 ? 0.2 : 0.0);
    P.integral_cutoff = c.integralCutoff;
    P.mixed_cut = c.mixed_cut;
    P.class_count32 = c.d_class_count32.p;
    P.class_end = c.d_pass_end.p ? c.d_pass_end.p + last : c.d_class_end.p;
    P.ket_segs = c.d_ket_segs.p;
    P.prim32 = c.d_prim32.p;
    P.pair_A = c.d_pair_A.p;
    P.boys32 = c.d_boys32.p;
    P.fixed_point = c.fixed_point;
    return P;
}

// Size the per-class quartet lists by the Schwarz-only count (an upper bound
// for every density), once per geometry and cutoff.
static double g_sized_cutoff = -1.0;

// Device memory the quartet lists of one pass may take: QB_LIST_BUDGET_MB,
// else 35% of the device memory free when the lists are sized.
static double list_budget_bytes(const Context& c)
{
    (void)c;
    const char* mb = getenv("QB_LIST_BUDGET_MB");
    if (mb && atof(mb) > 0) return atof(mb) * 1048576.0;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) != cudaSuccess) return 16.0 * 1073741824.0;
    return 0.35 * (double)fr;
}
static int size_quartet_lists(Context& c)
{
    CK(c.d_screen_cls.alloc(kNumClasses));
    CK(c.d_counts.alloc(kNumClasses));
    CK(c.d_counts32.alloc(kNumClasses));
    CK(c.d_class_count.alloc(kNumClasses));
    CK(c.d_class_count32.alloc(kNumClasses));
    CK(c.d_class_offset.alloc(kNumClasses));
    CK(c.d_class_end.alloc(kNumClasses));
    CK(c.d_overflow.alloc(1));
    CK(cudaMemcpy(c.d_screen_cls.p, c.screen_cls.data(), kNumClasses * sizeof(ScreenClass), cudaMemcpyHostToDevice));
    CK(cudaMemsetAsync(c.d_counts.p, 0, kNumClasses * sizeof(unsigned long long), c.stream));
    FockParams P = fock_params(c);
    ScreenParams S{c.d_screen_cls.p, c.d_counts.p, nullptr, c.d_counts32.p};
    launch_screen(S, P, kNumClasses, 1, c.nsm, c.stream);
    CK(cudaGetLastError());
    std::vector<unsigned long long> cnt(kNumClasses);
    CK(cudaMemcpyAsync(cnt.data(), c.d_counts.p, kNumClasses * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    long long off = 0;
    std::vector<long long> offs(kNumClasses), ends(kNumClasses);
    for (int k = 0; k < kNumClasses; k++) {
        c.screen_cls[k].out_offset = off;
        c.screen_cls[k].capacity = (long long)cnt[k];
        offs[k] = off;
        off += (long long)cnt[k];
        ends[k] = off;
    }
    CK(cudaMemcpy(c.d_screen_cls.p, c.screen_cls.data(), kNumClasses * sizeof(ScreenClass), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.d_class_offset.p, offs.data(), kNumClasses * sizeof(long long), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.d_class_end.p, ends.data(), kNumClasses * sizeof(long long), cudaMemcpyHostToDevice));
    // passes over disjoint bra ranges when the whole list would pass the
    // budget: each class's bra range cut into npass equal parts, counted
    // again per pass; npass doubles until the largest pass fits (or 64)
    const int K = kNumClasses;
    const double budget = list_budget_bytes(c);
    int npass = 1;
    long long longest = off;
    std::vector<ScreenClass> pc(c.screen_cls);
    if ((double)off * sizeof(Quartet) > budget) {
        npass = std::min(64, (int)std::ceil((double)off * sizeof(Quartet) / budget));
        std::vector<unsigned long long> pcnt;
        for (;;) {
            pc.assign((size_t)npass * K, ScreenClass{});
            for (int p = 0; p < npass; p++)
                for (int k = 0; k < K; k++) {
                    ScreenClass s = c.screen_cls[k];
                    const long long nb = s.bra_end - s.bra_begin;
                    s.bra_end = s.bra_begin + (int)(nb * (p + 1) / npass);
                    s.bra_begin = s.bra_begin + (int)(nb * p / npass);
                    pc[(size_t)p * K + k] = s;
                }
            CK(c.d_pass_cls.alloc(pc.size()));
            CK(cudaMemcpy(c.d_pass_cls.p, pc.data(), pc.size() * sizeof(ScreenClass), cudaMemcpyHostToDevice));
            pcnt.assign((size_t)npass * K, 0);
            longest = 0;
            for (int p = 0; p < npass; p++) {
                CK(cudaMemsetAsync(c.d_counts.p, 0, K * sizeof(unsigned long long), c.stream));
                ScreenParams Sp{c.d_pass_cls.p + (size_t)p * K, c.d_counts.p, nullptr, c.d_counts32.p};
                launch_screen(Sp, P, K, 1, c.nsm, c.stream);
                CK(cudaGetLastError());
                CK(cudaMemcpyAsync(pcnt.data() + (size_t)p * K, c.d_counts.p, K * sizeof(unsigned long long),
                                   cudaMemcpyDeviceToHost, c.stream));
            }
            CK(cudaStreamSynchronize(c.stream));
            for (int p = 0; p < npass; p++) {
                long long o = 0;
                for (int k = 0; k < K; k++) {
                    ScreenClass& s = pc[(size_t)p * K + k];
                    s.out_offset = o;
                    s.capacity = (long long)pcnt[(size_t)p * K + k];
                    o += s.capacity;
                }
                longest = std::max(longest, o);
            }
            if ((double)longest * sizeof(Quartet) <= budget || npass >= 64) break;
            npass = std::min(64, 2 * npass);
        }
    }
    c.npass = npass;
    c.pass_cls = pc;
    std::vector<long long> po((size_t)npass * K), pe((size_t)npass * K);
    for (size_t i = 0; i < pc.size(); i++) {
        po[i] = pc[i].out_offset;
        pe[i] = pc[i].out_offset + pc[i].capacity;
    }
    CK(c.d_pass_cls.alloc(pc.size()));
    CK(c.d_pass_offset.alloc(pc.size()));
    CK(c.d_pass_end.alloc(pc.size()));
    CK(c.d_total_count.alloc(K));
    CK(c.d_total_count32.alloc(K));
    CK(cudaMemcpy(c.d_pass_cls.p, pc.data(), pc.size() * sizeof(ScreenClass), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.d_pass_offset.p, po.data(), po.size() * sizeof(long long), cudaMemcpyHostToDevice));
    CK(cudaMemcpy(c.d_pass_end.p, pe.data(), pe.size() * sizeof(long long), cudaMemcpyHostToDevice));
    CK(c.d_quartets.alloc((size_t)std::max<long long>(longest, 1)));
    g_sized_cutoff = c.integralCutoff;
    return 0;
}

// Class counts of the last build, summed over its passes.
static const int* build_counts(const Context& c, int f32)
{
    if (c.npass > 1) return f32 ? c.d_total_count32.p : c.d_total_count.p;
    return f32 ? c.d_class_count32.p : c.d_class_count.p;
}

// Screening into the per-class quartet lists for the current density; the
// class counts come back to the host to size the class launches.
static int screen_quartets(Context& c, int pass, std::vector<int>& cnt, std::vector<int>& cnt32)
{
    if (require(c.have_pairs, "gpu_upload_cutoff_matrix_ must precede the two-electron kernels")) return 1;
    if (require(c.have_cutoff, "gpu_upload_cutoff_ must precede the two-electron kernels")) return 1;
    if (g_sized_cutoff != c.integralCutoff || c.d_quartets.p == nullptr)
        if (size_quartet_lists(c)) return 2;
    int n = c.nbasis;
    CK(cudaMemsetAsync(c.d_counts.p, 0, kNumClasses * sizeof(unsigned long long), c.stream));
    CK(cudaMemsetAsync(c.d_counts32.p, 0, kNumClasses * sizeof(unsigned long long), c.stream));
    CK(cudaMemsetAsync(c.d_overflow.p, 0, sizeof(int), c.stream));
    CK(c.d_dense.alloc((size_t)n * n));
    if (pass == 0) launch_scale_density(c.d_dense_raw.p, c.d_cons.p, c.d_dense.p, n, c.stream);
    FockParams P = fock_params(c);   // with the mixed split: the FP32 list from the back of each class region
    P.class_offset = c.d_pass_offset.p + (size_t)pass * kNumClasses;
    P.class_end = c.d_pass_end.p + (size_t)pass * kNumClasses;
    ScreenParams S{c.d_pass_cls.p + (size_t)pass * kNumClasses, c.d_counts.p, c.d_quartets.p, c.d_counts32.p};
    launch_screen(S, P, kNumClasses, 0, c.nsm, c.stream);
    launch_finish_counts(S, c.d_class_count.p, c.d_class_count32.p, c.d_overflow.p, kNumClasses, c.stream);
    CK(cudaGetLastError());
    cnt.assign(kNumClasses, 0);
    cnt32.assign(kNumClasses, 0);
    int ovf = 0;
    CK(cudaMemcpyAsync(cnt.data(), c.d_class_count.p, kNumClasses * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(cnt32.data(), c.d_class_count32.p, kNumClasses * sizeof(int), cudaMemcpyDeviceToHost,
                       c.stream));
    CK(cudaMemcpyAsync(&ovf, c.d_overflow.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    if (ovf) return set_error(3, "quartet list overflow (internal sizing error)"), 3;
    return 0;
}

// The classes are independent: their kernels are dealt round-robin to the
// library stream and up to kSideStreams side streams, forked from and joined
// back into the library stream with events (so a CUDA graph capture keeps
// the order), which fills the tail of one class's launch with the next.
// QB_CLASS_STREAMS sets the total number of streams (default 4).
static int fork_side_streams(Context& c)
{
    if (c.nside < 0) {
        const char* ns = getenv("QB_CLASS_STREAMS");
        c.nside = std::max(0, std::min(ns ? atoi(ns) - 1 : kSideStreams, kSideStreams));
        for (int i = 0; i < c.nside; i++) {
            CK(cudaStreamCreateWithFlags(&c.side[i], cudaStreamNonBlocking));
            CK(cudaEventCreateWithFlags(&c.side_ev[i], cudaEventDisableTiming));
        }
        CK(cudaEventCreateWithFlags(&c.fork_ev, cudaEventDisableTiming));
    }
    if (c.nside > 0) {
        CK(cudaEventRecord(c.fork_ev, c.stream));
        for (int i = 0; i < c.nside; i++) CK(cudaStreamWaitEvent(c.side[i], c.fork_ev, 0));
    }
    return 0;
}

static cudaStream_t side_stream(Context& c, int turn)
{
    const int t = turn % (c.nside + 1);
    return t == 0 ? c.stream : c.side[t - 1];
}

static int join_side_streams(Context& c)
{
    for (int i = 0; i < c.nside; i++) {
        CK(cudaEventRecord(c.side_ev[i], c.side[i]));
        CK(cudaStreamWaitEvent(c.stream, c.side_ev[i], 0));
    }
    return 0;
}

// Two-electron gradient into d_grad (3 natom), same quartet lists.
// Lanes per quartet of gradient class k (qb_autotune_grad's choice, else 1).
static int grad_lanes(const Context& c, int k, int f32)
{
    const std::vector<int>& g = f32 ? c.grad_group32 : c.grad_group;
    return g.empty() ? 1 : std::min(std::max(g[k], 1), grad_max_group(k));
}

static int grad_build(Context& c)
{
    std::vector<int> cnt, cnt32;
    if (require(c.have_pairs && c.have_cutoff, "gpu_upload_cutoff_ must precede the gradient")) return 1;
    if (g_sized_cutoff != c.integralCutoff || c.d_quartets.p == nullptr)
        if (size_quartet_lists(c)) return 2;
    CK(c.d_grad.alloc(3 * (size_t)c.natom));
    CK(cudaMemsetAsync(c.d_grad.p, 0, 3 * (size_t)c.natom * sizeof(double), c.stream));
    // per-block shared accumulation while 3 natom doubles fit the default 48 KB
    GradExtra G{c.d_shell_atom.p, c.d_pair_sh.p, c.d_grad.p, c.natom, 3 * c.natom * 8 <= 48 * 1024 ? 1 : 0};
    for (int k = 0; k < 4; k++)
        if (!c.ev[k]) CK(cudaEventCreate(&c.ev[k]));
    long long total = 0;
    for (int pass = 0; pass < c.npass; pass++) {
    if (int rc = screen_quartets(c, pass, cnt, cnt32)) return rc;
    FockParams P = fock_params(c);
    P.class_offset = c.d_pass_offset.p + (size_t)pass * kNumClasses;
    P.class_end = c.d_pass_end.p + (size_t)pass * kNumClasses;
    if (pass == 0) CK(cudaEventRecord(c.ev[2], c.stream));
    for (int k = 0; k < kNumClasses; k++) total += cnt[k] + cnt32[k];
    if (int rc = fork_side_streams(c)) return rc;
    int turn = 0;
    for (int k = 0; k < kNumClasses; k++)
        for (int f32 = 0; f32 < 2; f32++) {
            const int nq = f32 ? cnt32[k] : cnt[k];
            if (nq == 0) continue;
            const int GS = grad_lanes(c, k, f32);
            cudaStream_t st = side_stream(c, turn++);
            const int rc = f32 ? launch_grad_class32(k, P, G, GS, nq, c.nsm, st) : launch_grad_class(k, P, G, GS, nq, c.nsm, st);
            if (rc < 0) {
                // the generic kernels (FP64, either list) share one scratch
                // array: all on the library stream, in order
                const int* Lk = kClassL[k];
                if (launch_generic_grad_class(k, Lk[0], Lk[1], Lk[2], Lk[3], P, G, nq, c.nsm, f32, c.stream) < 0)
                    return set_error(2, "gpu_grad_: cannot allocate the scratch of class (%d%d|%d%d)", Lk[0], Lk[1],
                                     Lk[2], Lk[3]), 2;
            }
        }
    if (int rc = join_side_streams(c)) return rc;
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(c.ev[3], c.stream));
    CK(cudaStreamSynchronize(c.stream));
    float ms = 0.f;
    CK(cudaEventElapsedTime(&ms, c.ev[2], c.ev[3]));
    c.last_ms_grad = ms;
    c.last_grad_quartets = total;
    return 0;
}

// The Fock build proper, on device data already in place (d_dense,
// d_cut_matrix): screening, class kernels, O_out = O_in + G.
static int fock_build(Context& c, const double* d_o_in, double* d_o_out)
{
    if (require(c.have_pairs, "gpu_upload_cutoff_matrix_ must precede the Fock build")) return 1;
    if (require(c.have_cutoff, "gpu_upload_cutoff_ must precede the Fock build")) return 1;
    if (g_sized_cutoff != c.integralCutoff || c.d_quartets.p == nullptr)
        if (size_quartet_lists(c)) return 2;
    int n = c.nbasis;
    CK(c.d_fock.alloc((size_t)n * n));
    CK(cudaMemsetAsync(c.d_fock.p, 0, (size_t)n * n * sizeof(double), c.stream));
    CK(cudaMemsetAsync(c.d_counts.p, 0, kNumClasses * sizeof(unsigned long long), c.stream));
    CK(cudaMemsetAsync(c.d_counts32.p, 0, kNumClasses * sizeof(unsigned long long), c.stream));
    CK(cudaMemsetAsync(c.d_overflow.p, 0, sizeof(int), c.stream));
    CK(c.d_dense.alloc((size_t)n * n));
    launch_scale_density(c.d_dense_raw.p, c.d_cons.p, c.d_dense.p, n, c.stream);
    const int K = kNumClasses;
    for (int k = 0; k < 4; k++)
        if (!c.ev[k]) CK(cudaEventCreate(&c.ev[k]));
    if (c.npass > 1) {
        CK(cudaMemsetAsync(c.d_total_count.p, 0, K * sizeof(int), c.stream));
        CK(cudaMemsetAsync(c.d_total_count32.p, 0, K * sizeof(int), c.stream));
    }
    // one pass per bra range (one pass unless the lists pass the memory
    // budget); a pass's class kernels finish (join) before the next pass's
    // screen rewrites the shared list buffer
    for (int pass = 0; pass < c.npass; pass++) {
    FockParams P = fock_params(c);
    P.class_offset = c.d_pass_offset.p + (size_t)pass * K;
    P.class_end = c.d_pass_end.p + (size_t)pass * K;
    ScreenParams S{c.d_pass_cls.p + (size_t)pass * K, c.d_counts.p, c.d_quartets.p, c.d_counts32.p};
    if (pass > 0) {
        CK(cudaMemsetAsync(c.d_counts.p, 0, K * sizeof(unsigned long long), c.stream));
        CK(cudaMemsetAsync(c.d_counts32.p, 0, K * sizeof(unsigned long long), c.stream));
    }
    if (pass == 0) CK(cudaEventRecord(c.ev[0], c.stream));
    launch_screen(S, P, K, 0, c.nsm, c.stream);
    launch_finish_counts(S, c.d_class_count.p, c.d_class_count32.p, c.d_overflow.p, K, c.stream);
    if (c.npass > 1)
        launch_add_counts(c.d_class_count.p, c.d_class_count32.p, c.d_total_count.p, c.d_total_count32.p, K, c.stream);
    CK(cudaGetLastError());
    if (pass == 0) {
        CK(cudaEventRecord(c.ev[1], c.stream));
        CK(cudaEventRecord(c.ev[2], c.stream));
    }
    // The class kernels read their quartet counts on the device; the host
    // sizes their grids by the Schwarz-only capacity of each class (an upper
    // bound), so nothing between screening and digestion waits for the host
    // and the whole build can be captured in a CUDA graph.
    if (int rc = fork_side_streams(c)) return rc;
    int turn = 0;
    for (int k = 0; k < K; k++) {
        const long long cap = c.pass_cls[(size_t)pass * K + k].capacity;
        if (cap == 0) continue;
        const int nq = (int)std::min<long long>(cap, 1LL << 30);
        for (int f32 = 0; f32 < (c.mixed_cut > 0.0 ? 2 : 1); f32++) {
            const int G = f32 ? (c.class_group32.empty() ? 1 : c.class_group32[k])
                              : (c.class_group.empty() ? 1 : c.class_group[k]);
            const int* Lk = kClassL[k];
            const bool gen = Lk[0] + Lk[1] + Lk[2] + Lk[3] >= c.generic_min_l;
            cudaStream_t st = side_stream(c, turn++);
            const int rc = gen ? launch_generic_class(k, Lk[0], Lk[1], Lk[2], Lk[3], P, nq, c.nsm, f32, st)
                               : (f32 ? launch_class32(k, P, G, nq, c.nsm, st)
                                      : launch_class(k, P, G, nq, c.nsm, st));
            if (rc < 0)
                return set_error(5, "class (%d%d|%d%d) needs more shared memory than this GPU offers",
                                 kClassL[k][0], kClassL[k][1], kClassL[k][2], kClassL[k][3]), 5;
        }
    }
    if (int rc = join_side_streams(c)) return rc;
    }
    CK(cudaGetLastError());
    CK(cudaEventRecord(c.ev[3], c.stream));
    launch_fock_finish(c.d_fock.p, c.d_cons.p, d_o_in, d_o_out, n, c.stream, c.fixed_point);
    CK(cudaGetLastError());
    c.stats_pending = true;
    return 0;
}

// Counts, timings and the overflow flag of the last Fock build, read once
// it has finished (synchronises the library stream).
static int fock_stats_resolve(Context& c)
{
    if (!c.stats_pending) return 0;
    c.stats_pending = false;
    std::vector<int> cnt(kNumClasses), cnt32(kNumClasses);
    int ovf = 0;
    CK(cudaMemcpyAsync(cnt.data(), build_counts(c, 0), kNumClasses * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(cnt32.data(), build_counts(c, 1), kNumClasses * sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(&ovf, c.d_overflow.p, sizeof(int), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    if (ovf) return set_error(3, "quartet list overflow (internal sizing error)"), 3;
    long long total = 0, total32 = 0;
    for (int k = 0; k < kNumClasses; k++) total += cnt[k], total32 += cnt32[k];
    float ms0 = 0, ms1 = 0;
    CK(cudaEventElapsedTime(&ms0, c.ev[0], c.ev[1]));
    CK(cudaEventElapsedTime(&ms1, c.ev[2], c.ev[3]));
    c.last_ms_screen = ms0;
    c.last_ms_eri = ms1;
    c.last_quartets = total + total32;
    c.last_quartets32 = total32;
    return 0;
}

static Context& ctx()
{
    if (!g) g = new Context();
    return *g;
}

// Lanes per quartet of the gradient kernels of class k for the batched gradient (the session's choice).
int session_grad_lanes(int k, int f32)
{
    return grad_lanes(ctx(), k, f32);
}

}  // namespace qb

using namespace qb;

extern "C" {

int qb_status(void) { return g_status; }
const char* qb_last_error(void) { return g_err.c_str(); }
void qb_clear_error(void)
{
    g_status = 0;
    g_err.clear();
}

void gpu_startup_(void)
{
    delete g;
    g = new Context();
}

void gpu_set_device_(int* gpu_dev_id) { ctx().dev_id = *gpu_dev_id; }

void gpu_init_(void)
{
    Context& c = ctx();
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        set_error(10, "no CUDA device available (%s)", cudaGetErrorString(e));
        return;
    }
    int dev = c.dev_id < 0 ? 0 : c.dev_id;
    if (dev >= count) {
        set_error(11, "GPU id %d is illegal, select from 0 to %d", dev, count - 1);
        return;
    }
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, dev);
    if (prop.major < 10) {
        set_error(12, "device %d is sm_%d%d; this build targets sm_100a (B200)", dev, prop.major, prop.minor);
        return;
    }
    if (cudaSetDevice(dev) != cudaSuccess) {
        set_error(13, "cudaSetDevice(%d) failed", dev);
        return;
    }
    c.dev_id = dev;
    c.nsm = prop.multiProcessorCount;
    if (!c.own_stream) cudaStreamCreateWithFlags(&c.own_stream, cudaStreamNonBlocking);
    if (!c.stream) c.stream = c.own_stream;
    std::vector<double> tab;
    boys_table(tab);
    std::vector<float> tab32;
    boys_table32(tab32);
    if (c.d_boys.alloc(tab.size()) != cudaSuccess ||
        cudaMemcpy(c.d_boys.p, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess ||
        c.d_boys32.alloc(tab32.size()) != cudaSuccess ||
        cudaMemcpy(c.d_boys32.p, tab32.data(), tab32.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) {
        set_error(2, "cannot upload the Boys table");
        return;
    }
    c.inited = true;
}

int qb_set_stream(void* stream)
{
    Context& c = ctx();
    c.stream = stream ? (cudaStream_t)stream : c.own_stream;
    return 0;
}

void gpu_shutdown_(void)
{
    if (!g) return;
    Context& c = *g;
    DevBuf<double>* dbl[] = {&c.d_pair_Y, &c.d_boys, &c.d_dense, &c.d_dense_raw, &c.d_cons, &c.d_fock, &c.d_cut_matrix, &c.d_o_in, &c.d_o_out, &c.d_grad};
    c.d_shell_atom.release();
    for (auto* b : dbl) b->release();
    c.d_prim.release();
    c.d_prim32.release();
    c.d_pair_A.release();
    c.d_boys32.release();
    c.d_pair_bf.release();
    c.d_pair_sh.release();
    c.d_pair_AB.release();
    c.d_screen_cls.release();
    c.d_counts.release();
    c.d_counts32.release();
    c.d_class_count.release();
    c.d_class_count32.release();
    c.d_overflow.release();
    c.d_class_offset.release();
    c.d_class_end.release();
    c.d_pass_cls.release();
    c.d_pass_offset.release();
    c.d_pass_end.release();
    c.d_total_count.release();
    c.d_total_count32.release();
    c.npass = 1;
    c.pass_cls.clear();
    c.d_quartets.release();
    c.d_ket_segs.release();
    for (auto& e : c.ev)
        if (e) cudaEventDestroy(e), e = nullptr;
    for (int i = 0; i < c.nside; i++) {
        cudaStreamDestroy(c.side[i]);
        cudaEventDestroy(c.side_ev[i]);
    }
    if (c.fork_ev) cudaEventDestroy(c.fork_ev);
    xc_release();
    oneint_release();
    generic_release();
    noalloc_reset();
    batch_release();
    c.d_S1.release();
    c.d_H1.release();
    c.d_D1.release();
    c.d_W1.release();
    c.d_o_up.release();
    c.d_dense_up.release();
    c.sw_prim.release();
    c.sw_ab.release();
    c.sw_bf.release();
    c.sw_oc.release();
    c.sw_op.release();
    c.d_g1.release();
    c.d_shell_first.release();
    if (c.own_stream) cudaStreamDestroy(c.own_stream);
    delete g;
    g = nullptr;
    g_sized_cutoff = -1.0;
}

void gpu_get_device_info_(int* gpu_dev_count, int* gpu_dev_id, int* gpu_dev_mem, int* gpu_num_proc, double* gpu_core_freq,
                          char* gpu_dev_name, int* name_len, int* majorv, int* minorv)
{
    Context& c = ctx();
    *gpu_dev_id = c.dev_id;
    if (cudaGetDeviceCount(gpu_dev_count) != cudaSuccess || *gpu_dev_count == 0) {
        *gpu_dev_count = 0;
        set_error(10, "no CUDA device found");
        return;
    }
    cudaDeviceProp prop;
    cudaGetDeviceProperties(&prop, c.dev_id < 0 ? 0 : c.dev_id);
    *gpu_dev_mem = (int)(prop.totalGlobalMem / (1024 * 1024));
    *gpu_num_proc = prop.multiProcessorCount;
    int clk = 0;
    cudaDeviceGetAttribute(&clk, cudaDevAttrClockRate, c.dev_id < 0 ? 0 : c.dev_id);
    *gpu_core_freq = clk * 1e-6;
    strcpy(gpu_dev_name, prop.name);
    *name_len = (int)strlen(gpu_dev_name);
    *majorv = prop.major;
    *minorv = prop.minor;
}

void gpu_setup_(int* natom, int* nbasis, int* nElec, int* imult, int* molchg, int* iAtomType)
{
    Context& c = ctx();
    c.natom = *natom;
    c.nbasis = *nbasis;
    c.nelec = *nElec;
    c.imult = *imult;
    c.molchg = *molchg;
    c.iAtomType = *iAtomType;
}

void gpu_upload_method_(int* quick_method)
{
    if (*quick_method < 0 || *quick_method > 2) {
        set_error(1, "unknown method %d", *quick_method);
        return;
    }
    ctx().method = *quick_method;
}

void gpu_upload_xyz_(double* atom_xyz)
{
    Context& c = ctx();
    c.xyz.assign(atom_xyz, atom_xyz + 3 * c.natom);
    c.geom_version = ++g_geom_counter;
}

void gpu_upload_atom_and_chg_(int* atom, double* atom_chg)
{
    Context& c = ctx();
    c.iattype.assign(atom, atom + c.natom);
    c.chg.assign(atom_chg, atom_chg + c.natom);
    c.geom_version = ++g_geom_counter;
}

void gpu_upload_basis_(int* nshell, int* nprim, int* jshell, int* jbasis, int* maxcontract, int* ncontract, int* itype,
                       double* aexp, double* dcoeff, int* first_basis_function, int* last_basis_function,
                       int* first_shell_basis_function, int* last_shell_basis_function, int* ncenter, int* kstart,
                       int* katom, int* ktype, int* kprim, int* kshell, int* Ksumtype, int* Qnumber, int* Qstart,
                       int* Qfinal, int* Qsbasis, int* Qfbasis, double* gccoeff, double* cons, double* gcexpo, int* KLMN)
{
    Context& c = ctx();
    c.nshell = *nshell;
    c.nprim = *nprim;
    c.jshell = *jshell;
    c.jbasis = *jbasis;
    c.maxcontract = *maxcontract;
    int ns = c.nshell, nb = c.nbasis;
    c.kstart.assign(kstart, kstart + ns);
    c.katom.assign(katom, katom + ns);
    c.kprim.assign(kprim, kprim + ns);
    c.Ksumtype.assign(Ksumtype, Ksumtype + ns + 1);
    c.Qnumber.assign(Qnumber, Qnumber + ns);
    c.Qstart.assign(Qstart, Qstart + ns);
    c.Qfinal.assign(Qfinal, Qfinal + ns);
    c.Qsbasis.assign(Qsbasis, Qsbasis + 4 * ns);
    c.Qfbasis.assign(Qfbasis, Qfbasis + 4 * ns);
    c.KLMN.assign(KLMN, KLMN + 3 * nb);
    c.gccoeff.assign(gccoeff, gccoeff + (size_t)MAXPRIM * nb);
    c.gcexpo.assign(gcexpo, gcexpo + (size_t)MAXPRIM * nb);
    c.cons.assign(cons, cons + nb);
    c.ncontract.assign(ncontract, ncontract + nb);
    c.itype.assign(itype, itype + 3 * nb);
    c.ncenter.assign(ncenter, ncenter + nb);
    c.aexp.assign(aexp, aexp + (size_t)c.maxcontract * nb);
    c.dcoeff.assign(dcoeff, dcoeff + (size_t)c.maxcontract * nb);
    c.geom_version = ++g_geom_counter;
    (void)first_basis_function; (void)last_basis_function;
    (void)first_shell_basis_function; (void)last_shell_basis_function; (void)ktype; (void)kshell;
    for (int s = 0; s < ns; s++) {
        if (c.kprim[s] < 1 || c.kprim[s] > MAXPRIM) {
            set_error(1, "shell %d has %d primitives (1..%d supported)", s + 1, c.kprim[s], MAXPRIM);
            return;
        }
        if (c.Qstart[s] < 0 || c.Qfinal[s] > 3 || c.Qfinal[s] < c.Qstart[s]) {
            set_error(1, "shell %d has angular momentum %d..%d (s..f supported)", s + 1, c.Qstart[s], c.Qfinal[s]);
            return;
        }
    }
    // The generated kernels emit Cartesian components in QUICK's KLMN order
    // (src/basis.f90:546-643); refuse any other order.
    static const int order[4][10][3] = {
        {{0, 0, 0}},
        {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}},
        {{2, 0, 0}, {1, 1, 0}, {0, 2, 0}, {1, 0, 1}, {0, 1, 1}, {0, 0, 2}},
        {{3, 0, 0}, {2, 1, 0}, {1, 2, 0}, {0, 3, 0}, {2, 0, 1}, {1, 1, 1}, {0, 2, 1}, {1, 0, 2}, {0, 1, 2}, {0, 0, 3}}};
    for (int s = 0; s < ns; s++)
        for (int L = c.Qstart[s]; L <= c.Qfinal[s]; L++) {
            int f0 = bf_first(c, s, L);
            for (int k = 0; k < (L + 1) * (L + 2) / 2; k++)
                for (int x = 0; x < 3; x++)
                    if (c.KLMN[3 * (f0 + k) + x] != order[L][k][x]) {
                        set_error(1, "basis function %d: Cartesian order differs from QUICK's", f0 + k + 1);
                        return;
                    }
        }
    sort_qshells(c);
    if (c.d_cons.alloc(nb) != cudaSuccess ||
        cudaMemcpy(c.d_cons.p, c.cons.data(), nb * sizeof(double), cudaMemcpyHostToDevice) != cudaSuccess) {
        set_error(2, "cannot upload cons");
        return;
    }
    c.have_basis = true;
    c.have_pairs = false;
}

void gpu_upload_cutoff_matrix_(double* YCutoff, double* cutPrim)
{
    Context& c = ctx();
    if (require(c.have_basis, "gpu_upload_basis_ must precede gpu_upload_cutoff_matrix_")) return;
    if (require(c.inited, "gpu_init_ must precede gpu_upload_cutoff_matrix_")) return;
    c.YCutoff.assign(YCutoff, YCutoff + (size_t)c.nshell * c.nshell);
    c.cutPrim.assign(cutPrim, cutPrim + (size_t)c.jbasis * c.jbasis);
    build_pairlist(c.Qshell, c.sorted_Q.data(), c.sorted_Qnumber.data(), c.kprim.data(), c.nshell, c.YCutoff.data(), c.ref_xy,
                   c.fStart, c.ffStart);
    if (build_tables(c)) return;
    g_sized_cutoff = -1.0;
    c.have_pairs = true;
}

// Copies O and the density to the device at the call (QUICK copies them at
// this call too, gpu.cu): straight from the caller's arrays, one DMA each
// when the caller's memory is pinned; the call returns once both are copied,
// so the caller may reuse its arrays.
void gpu_upload_calculated_(double* o, double* co, double* vec, double* dense)
{
    (void)co;
    (void)vec;
    Context& c = ctx();
    size_t nn = (size_t)c.nbasis * c.nbasis;
    if (c.d_o_up.alloc(nn) != cudaSuccess || c.d_dense_up.alloc(nn) != cudaSuccess ||
        cudaMemcpyAsync(c.d_o_up.p, o, nn * sizeof(double), cudaMemcpyHostToDevice, c.stream) != cudaSuccess ||
        cudaMemcpyAsync(c.d_dense_up.p, dense, nn * sizeof(double), cudaMemcpyHostToDevice, c.stream) != cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess) {
        set_error(2, "upload of the density / operator failed");
        return;
    }
    c.o_host_valid = false;
    c.have_calc = true;
}

// The uploaded O on the host (for the paths that add to it there).
static const std::vector<double>& host_o(Context& c)
{
    if (!c.o_host_valid) {
        const size_t nn = (size_t)c.nbasis * c.nbasis;
        c.o_host.resize(nn);
        if (cudaMemcpyAsync(c.o_host.data(), c.d_o_up.p, nn * sizeof(double), cudaMemcpyDeviceToHost, c.stream) ==
                cudaSuccess &&
            cudaStreamSynchronize(c.stream) == cudaSuccess)
            c.o_host_valid = true;
        else
            set_error(2, "download of the uploaded operator failed");
    }
    return c.o_host;
}

void gpu_upload_cutoff_(double* cutMatrix, double* integralCutoff, double* primLimit, double* DMCutoff)
{
    (void)DMCutoff;   // never read: Fortran callers pass three arguments
    Context& c = ctx();
    c.integralCutoff = *integralCutoff;
    c.primLimit = *primLimit;
    c.DMCutoff = 1e-9;
    c.cutMatrix.assign(cutMatrix, cutMatrix + (size_t)c.nshell * c.nshell);
    if (c.d_cut_matrix.alloc(c.cutMatrix.size()) != cudaSuccess ||
        cudaMemcpyAsync(c.d_cut_matrix.p, c.cutMatrix.data(), c.cutMatrix.size() * sizeof(double), cudaMemcpyHostToDevice,
                        c.stream) != cudaSuccess) {
        set_error(2, "cannot upload cutMatrix");
        return;
    }
    c.have_cutoff = true;
}

void gpu_get2e_(double* o)
{
    Context& c = ctx();
    if (require(c.have_calc, "gpu_upload_calculated_ must precede gpu_get2e_")) return;
    size_t nn = (size_t)c.nbasis * c.nbasis;
    if (c.d_dense_raw.alloc(nn) != cudaSuccess || c.d_o_in.alloc(nn) != cudaSuccess || c.d_o_out.alloc(nn) != cudaSuccess) {
        set_error(2, "cannot allocate %zu-element matrices", nn);
        return;
    }
    if (cudaMemcpyAsync(c.d_dense_raw.p, c.d_dense_up.p, nn * sizeof(double), cudaMemcpyDeviceToDevice, c.stream) != cudaSuccess ||
        cudaMemcpyAsync(c.d_o_in.p, c.d_o_up.p, nn * sizeof(double), cudaMemcpyDeviceToDevice, c.stream) != cudaSuccess) {
        set_error(2, "copy of density / operator failed");
        return;
    }
    if (fock_build(c, c.d_o_in.p, c.d_o_out.p)) return;
    if (cudaMemcpyAsync(o, c.d_o_out.p, nn * sizeof(double), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess) {
        set_error(2, "download of the operator failed");
        return;
    }
    fock_stats_resolve(c);
}

int qb_fock_device(const double* d_dense, const double* d_o_in, double* d_o_out)
{
    Context& c = ctx();
    size_t nn = (size_t)c.nbasis * c.nbasis;
    CK(c.d_dense_raw.alloc(nn));
    CK(cudaMemcpyAsync(c.d_dense_raw.p, d_dense, nn * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
    return fock_build(c, d_o_in, d_o_out);
}

// Gradient counterpart of qb_autotune_classes: after a gradient call, every
// compiled lanes-per-quartet size of every gradient class with more than one
// (the light classes) is timed on that call's quartet lists into a scratch
// gradient, and the fastest is kept for the session's later gradients (the
// FP32 kernels after a call with the mixed split).
int qb_autotune_grad(int* groups, int cap)
{
    Context& c = ctx();
    if (require(c.have_pairs && c.have_cutoff && c.d_quartets.p != nullptr && c.natom > 0,
                "a gradient call must precede qb_autotune_grad"))
        return 1;
    DevBuf<double> scratch;
    CK(scratch.alloc(3 * (size_t)c.natom));
    CK(cudaMemsetAsync(scratch.p, 0, 3 * (size_t)c.natom * sizeof(double), c.stream));
    FockParams P = fock_params(c);
    GradExtra G{c.d_shell_atom.p, c.d_pair_sh.p, scratch.p, c.natom, 3 * c.natom * 8 <= 48 * 1024 ? 1 : 0};
    const bool verbose = getenv("QB_AUTOTUNE_VERBOSE") && atoi(getenv("QB_AUTOTUNE_VERBOSE")) > 0;
    std::vector<int> cnt(kNumClasses), cnt32(kNumClasses);
    CK(cudaMemcpy(cnt.data(), c.d_class_count.p, kNumClasses * sizeof(int), cudaMemcpyDeviceToHost));
    CK(cudaMemcpy(cnt32.data(), c.d_class_count32.p, kNumClasses * sizeof(int), cudaMemcpyDeviceToHost));
    const bool f32 = c.mixed_cut > 0.0;
    std::vector<int>& gg = f32 ? c.grad_group32 : c.grad_group;
    if (gg.empty()) gg.assign(kNumClasses, 1);
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    for (int k = 0; k < kNumClasses; k++) {
        const int nq = f32 ? cnt32[k] : cnt[k];
        if (nq == 0 || grad_max_group(k) < 2) continue;
        int best_g = gg[k];
        float best_t = 1e30f;
        for (int g = 1; g <= grad_max_group(k); g *= 2) {
            float tmin = 1e30f;
            for (int rep = 0; rep < 2; rep++) {
                CK(cudaEventRecord(e0, c.stream));
                const int rc = f32 ? launch_grad_class32(k, P, G, g, nq, c.nsm, c.stream)
                                   : launch_grad_class(k, P, G, g, nq, c.nsm, c.stream);
                CK(cudaEventRecord(e1, c.stream));
                CK(cudaEventSynchronize(e1));
                if (rc < 0) break;
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, e0, e1));
                tmin = std::min(tmin, ms);
            }
            if (verbose)
                fprintf(stderr, "autotune grad %s (%d%d|%d%d) GS=%d %.4f ms\n", f32 ? "fp32" : "fp64", kClassL[k][0],
                        kClassL[k][1], kClassL[k][2], kClassL[k][3], g, tmin);
            if (tmin < best_t) best_t = tmin, best_g = g;
        }
        gg[k] = best_g;
    }
    CK(cudaGetLastError());
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    scratch.release();
    for (int k = 0; k < std::min(cap, kNumClasses); k++) groups[k] = gg[k];
    return 0;
}

// Sets the lanes per quartet of every gradient class, as if tuned: each
// must be a compiled size (a power of two up to the class's maximum).
int qb_set_grad_groups(const int* groups, int n, int fp32)
{
    Context& c = ctx();
    if (require(n == kNumClasses, "qb_set_grad_groups: one size per class expected")) return 1;
    for (int k = 0; k < n; k++) {
        const int g = groups[k];
        if (g < 1 || g > grad_max_group(k) || (g & (g - 1))) {
            set_error(1, "qb_set_grad_groups: %d lanes is not compiled for class %d", g, k);
            return 1;
        }
    }
    (fp32 ? c.grad_group32 : c.grad_group).assign(groups, groups + n);
    return 0;
}

// Bra-range passes of the current quartet lists (1 unless the lists pass the
// memory budget).
int qb_list_passes(void)
{
    return ctx().npass;
}

// The launch variants of class cls (codes as qb_autotune_classes writes them).
int qb_class_variants(int cls, int fp32, int* codes, int cap)
{
    if (cls < 0 || cls >= kNumClasses) return 0;
    return class_variants(cls, fp32 ? 1 : 0, codes, cap);
}

// Sets the launch variant of every class (the codes qb_autotune_classes
// writes), as if tuned: each code must be one of the class's variants.
int qb_set_class_groups(const int* groups, int n, int fp32)
{
    Context& c = ctx();
    if (require(c.have_basis, "gpu_upload_basis_ must precede qb_set_class_groups")) return 1;
    if (require(n == kNumClasses, "qb_set_class_groups: one code per class expected")) return 1;
    std::vector<int> v(groups, groups + n);
    for (int k = 0; k < n; k++) {
        int codes[16];
        const int nv = class_variants(k, fp32 ? 1 : 0, codes, 16);
        bool ok = false;
        for (int i = 0; i < nv; i++) ok = ok || codes[i] == v[k];
        if (!ok) {
            set_error(1, "qb_set_class_groups: code %d is not a variant of class %d", v[k], k);
            return 1;
        }
    }
    (fp32 ? c.class_group32 : c.class_group) = v;
    (fp32 ? c.tuned32 : c.tuned64) = true;
    return 0;
}

// Per-class autotuning of the lanes per shell quartet: after a Fock build,
// every compiled variant of every straight-line class (each lane-group size,
// and for the light classes the kernels that stage the Boys records in
// shared memory, code kSbFlag + lanes) is timed on that build's quartet
// lists (writing into a scratch Fock matrix), and the fastest is kept for
// the following builds of the session.
int qb_autotune_classes(int* groups, int cap)
{
    Context& c = ctx();
    if (require(c.have_pairs && c.have_cutoff && c.d_quartets.p != nullptr,
                "a Fock build must precede qb_autotune_classes"))
        return 1;
    const int n = c.nbasis;
    DevBuf<double> scratch;
    CK(scratch.alloc((size_t)n * n));
    CK(cudaMemsetAsync(scratch.p, 0, (size_t)n * n * sizeof(double), c.stream));
    FockParams P = fock_params(c);
    P.fock = scratch.p;
    const bool verbose = getenv("QB_AUTOTUNE_VERBOSE") && atoi(getenv("QB_AUTOTUNE_VERBOSE")) > 0;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    // the last build's lists: its FP64 kernels are tuned after an all-FP64
    // build, its FP32 kernels after a build with the mixed split
    std::vector<int> cnt32(kNumClasses);
    CK(cudaMemcpy(cnt32.data(), c.d_class_count32.p, kNumClasses * sizeof(int), cudaMemcpyDeviceToHost));
    const bool f32 = c.mixed_cut > 0.0;
    std::vector<int>& groups_k = f32 ? c.class_group32 : c.class_group;
    for (int k = 0; k < kNumClasses; k++) {
        const long long capk = c.screen_cls[k].capacity;
        const int* Lk = kClassL[k];
        if (capk == 0 || Lk[0] + Lk[1] + Lk[2] + Lk[3] >= c.generic_min_l || kClassGeneric[k]) continue;
        if (f32 && cnt32[k] == 0) continue;
        const int nq = (int)std::min<long long>(capk, 1LL << 30);
        int best_g = groups_k[k];
        float best_t = 1e30f;
        int codes[16];
        const int nv = class_variants(k, f32 ? 1 : 0, codes, 16);
        for (int vi = 0; vi < nv; vi++) {
            const int g = codes[vi];
            float tmin = 1e30f;
            for (int rep = 0; rep < 2; rep++) {
                CK(cudaEventRecord(e0, c.stream));
                if (f32) launch_class32(k, P, g, nq, c.nsm, c.stream);
                else launch_class(k, P, g, nq, c.nsm, c.stream);
                CK(cudaEventRecord(e1, c.stream));
                CK(cudaEventSynchronize(e1));
                float ms = 0.f;
                CK(cudaEventElapsedTime(&ms, e0, e1));
                tmin = std::min(tmin, ms);
            }
            if (verbose)
                fprintf(stderr, "autotune %s (%d%d|%d%d) G=%d %.4f ms\n", f32 ? "fp32" : "fp64", Lk[0], Lk[1], Lk[2],
                        Lk[3], g, tmin);
            if (tmin < best_t) best_t = tmin, best_g = g;
        }
        groups_k[k] = best_g;
    }
    (f32 ? c.tuned32 : c.tuned64) = true;
    CK(cudaGetLastError());
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    scratch.release();
    for (int k = 0; k < std::min(cap, kNumClasses); k++) groups[k] = groups_k[k];
    return 0;
}

int qb_upload_cutoff_device(const double* d_dense, double integralCutoff, double primLimit)
{
    Context& c = ctx();
    if (require(c.have_basis, "gpu_upload_basis_ must precede qb_upload_cutoff_device")) return 1;
    c.integralCutoff = integralCutoff;
    c.primLimit = primLimit;
    c.DMCutoff = 1e-9;
    const size_t ns = c.nshell;
    CK(c.d_cut_matrix.alloc(ns * ns));
    if (c.shell_first_version != c.geom_version || !c.d_shell_first.p) {
        std::vector<int> first(ns + 1);
        for (size_t s = 0; s <= ns; s++) first[s] = c.Ksumtype[s] - 1;
        CK(c.d_shell_first.alloc(ns + 1));
        CK(cudaMemcpy(c.d_shell_first.p, first.data(), (ns + 1) * sizeof(int), cudaMemcpyHostToDevice));
        c.shell_first_version = c.geom_version;
    }
    launch_density_screen(d_dense, c.d_shell_first.p, (int)ns, c.nbasis, c.d_cut_matrix.p, c.stream);
    CK(cudaGetLastError());
    c.have_cutoff = true;
    return 0;
}

int qb_grad_device(const double* d_dense, double* d_grad)
{
    Context& c = ctx();
    if (require(c.have_pairs && c.have_cutoff, "the pair list and cutoffs must be uploaded before qb_grad_device")) return 1;
    const size_t nn = (size_t)c.nbasis * c.nbasis;
    CK(c.d_dense_raw.alloc(nn));
    CK(cudaMemcpyAsync(c.d_dense_raw.p, d_dense, nn * sizeof(double), cudaMemcpyDeviceToDevice, c.stream));
    if (int rc = grad_build(c)) return rc;
    launch_add_vector(c.d_grad.p, d_grad, 3 * c.natom, c.stream);
    CK(cudaGetLastError());
    return 0;
}

int qb_xc_grad_device(const double* d_dense, const double* sigrad2, double* d_grad)
{
    Context& c = ctx();
    if (require(c.have_basis && !c.xyz.empty(), "basis and coordinates must be uploaded before qb_xc_grad_device"))
        return 1;
    XcInputs in;
    in.natom = c.natom;
    in.nbasis = c.nbasis;
    in.maxcontract = c.maxcontract;
    in.method = c.method;
    in.xyz = c.xyz.data();
    in.iattype = c.iattype.data();
    in.ncenter = c.ncenter.data();
    in.itype = c.itype.data();
    in.ncontract = c.ncontract.data();
    in.aexp = c.aexp.data();
    in.dcoeff = c.dcoeff.data();
    in.sigrad2 = sigrad2;
    in.geom_version = c.geom_version;
    in.grid = c.xc_grid;
    in.stream = c.stream;
    double ms = 0.0;
    if (int rc = xc_gradient(in, d_dense, d_grad, &ms)) return rc;
    c.last_ms_xc_grad = ms;
    return 0;
}

int qb_set_fixed_point(int on)
{
    Context& c = ctx();
    c.fixed_point = on ? 1 : 0;
    return 0;
}

int qb_set_xc_grid(int grid)
{
    Context& c = ctx();
    if (grid != 1 && grid != 2) return set_error(1, "qb_set_xc_grid: grid must be 1 (SG1) or 2 (75 x 302 Becke)"), 1;
    c.xc_grid = grid;
    return 0;
}

int qb_xc_device(const double* d_dense, const double* sigrad2, double* d_vxc, double* exc, double* nalpha)
{
    Context& c = ctx();
    if (require(c.have_basis && !c.xyz.empty(), "basis and coordinates must be uploaded before qb_xc_device")) return 1;
    XcInputs in;
    in.natom = c.natom;
    in.nbasis = c.nbasis;
    in.maxcontract = c.maxcontract;
    in.method = c.method;
    in.xyz = c.xyz.data();
    in.iattype = c.iattype.data();
    in.ncenter = c.ncenter.data();
    in.itype = c.itype.data();
    in.ncontract = c.ncontract.data();
    in.aexp = c.aexp.data();
    in.dcoeff = c.dcoeff.data();
    in.sigrad2 = sigrad2;
    in.geom_version = c.geom_version;
    in.grid = c.xc_grid;
    in.stream = c.stream;
    XcResult r;
    if (int rc = xc_quadrature(in, d_dense, d_vxc, &r)) return rc;
    c.last_xc = r;
    *exc = r.exc;
    *nalpha = r.nalpha;
    return 0;
}

static OneIntHost oneint_host(const Context& c)
{
    OneIntHost h{};
    h.natom = c.natom;
    h.nbasis = c.nbasis;
    h.nshell = c.nshell;
    h.maxcontract = c.maxcontract;
    h.xyz = c.xyz.data();
    h.chg = c.chg.data();
    h.kprim = c.kprim.data();
    h.katom = c.katom.data();
    h.Ksumtype = c.Ksumtype.data();
    h.Qstart = c.Qstart.data();
    h.Qfinal = c.Qfinal.data();
    h.Qsbasis = c.Qsbasis.data();
    h.itype = c.itype.data();
    h.KLMN = c.KLMN.data();
    h.aexp = c.aexp.data();
    h.dcoeff = c.dcoeff.data();
    h.gccoeff = c.gccoeff.data();
    h.gcexpo = c.gcexpo.data();
    h.cons = c.cons.data();
    h.d_boys = c.d_boys.p;
    h.geom_version = c.geom_version;
    h.nsm = c.nsm;
    h.stream = c.stream;
    return h;
}

static int oneint_ready(const Context& c, const char* who)
{
    char msg[160];
    snprintf(msg, sizeof msg, "basis, coordinates and charges must be uploaded before %s", who);
    return require(c.inited && c.have_basis && (int)c.xyz.size() == 3 * c.natom && (int)c.chg.size() == c.natom, msg);
}

int qb_oneint_device(double* d_S, double* d_H)
{
    Context& c = ctx();
    if (oneint_ready(c, "qb_oneint_device")) return 1;
    return oneint_run(oneint_host(c), d_S, d_H);
}

int qb_grad1e_device(const double* d_dense, const double* d_wdense, double* d_grad)
{
    Context& c = ctx();
    if (oneint_ready(c, "qb_grad1e_device")) return 1;
    return grad1e_run(oneint_host(c), d_dense, d_wdense, d_grad);
}

// Host-pointer forms: the matrices of fullx (S, quick_one_electron_integral.f90:31-46)
// and get1e (H = T + V, :1699-1809).
static int oneint_host_call(double* S, double* H, const char* who)
{
    Context& c = ctx();
    if (oneint_ready(c, who)) return 1;
    const size_t nn = (size_t)c.nbasis * c.nbasis;
    if (S) CK(c.d_S1.alloc(nn));
    if (H) CK(c.d_H1.alloc(nn));
    if (int rc = oneint_run(oneint_host(c), S ? c.d_S1.p : nullptr, H ? c.d_H1.p : nullptr)) return rc;
    if (S) CK(cudaMemcpyAsync(S, c.d_S1.p, nn * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    if (H) CK(cudaMemcpyAsync(H, c.d_H1.p, nn * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return 0;
}

int gpu_get1e_(double* o) { return oneint_host_call(nullptr, o, "gpu_get1e_"); }

int gpu_get_overlap_(double* s) { return oneint_host_call(s, nullptr, "gpu_get_overlap_"); }

int gpu_grad1e_(double* grad, const double* dense, const double* wdense)
{
    Context& c = ctx();
    if (oneint_ready(c, "gpu_grad1e_")) return 1;
    const size_t nn = (size_t)c.nbasis * c.nbasis, ng = 3 * (size_t)c.natom;
    CK(c.d_D1.alloc(nn));
    CK(c.d_W1.alloc(nn));
    CK(c.d_g1.alloc(ng));
    CK(cudaMemcpyAsync(c.d_D1.p, dense, nn * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    CK(cudaMemcpyAsync(c.d_W1.p, wdense, nn * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    CK(cudaMemcpyAsync(c.d_g1.p, grad, ng * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    if (int rc = grad1e_run(oneint_host(c), c.d_D1.p, c.d_W1.p, c.d_g1.p)) return rc;
    CK(cudaMemcpyAsync(grad, c.d_g1.p, ng * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    return 0;
}

int qb_last_xc_stats(long long* npts, long long* nchunks, double* ms, double* ms_grid)
{
    Context& c = ctx();
    *npts = c.last_xc.npts;
    *nchunks = c.last_xc.nchunks;
    *ms = c.last_xc.ms;
    *ms_grid = c.last_xc.ms_grid;
    return 0;
}

int qb_last_xc_work(double* bytes, double* flops, double* gemm_flops)
{
    Context& c = ctx();
    *bytes = c.last_xc.alg_bytes;
    *flops = c.last_xc.alg_flops;
    *gemm_flops = c.last_xc.gemm_flops;
    return 0;
}

long long qb_xc_grid(double* xyzw, long long cap) { return xc_grid_points(xyzw, cap); }

int qb_xc_functional(int method, int n, const double* rho, const double* sigma, double* out)
{
    Context& c = ctx();
    if (require(c.inited, "gpu_init_ must precede qb_xc_functional")) return 1;
    if (n <= 0) return 0;
    DevBuf<double> r, s, o;
    CK(r.alloc(n));
    CK(s.alloc(n));
    CK(o.alloc(3 * (size_t)n));
    CK(cudaMemcpyAsync(r.p, rho, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    CK(cudaMemcpyAsync(s.p, sigma, n * sizeof(double), cudaMemcpyHostToDevice, c.stream));
    int rc = xc_functional_device(method, n, r.p, s.p, o.p, c.stream);
    if (!rc) {
        CK(cudaMemcpyAsync(out, o.p, 3 * (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
        CK(cudaStreamSynchronize(c.stream));
    }
    r.release();
    s.release();
    o.release();
    return rc;
}

int qb_last_grad_stats(long long* quartets, double* ms)
{
    Context& c = ctx();
    *quartets = c.last_grad_quartets;
    *ms = c.last_ms_grad;
    return 0;
}

int qb_set_mixed_precision(double cut)
{
    if (!(cut >= 0.0)) return set_error(1, "qb_set_mixed_precision: cut must be >= 0"), 1;
    ctx().mixed_cut = cut;
    return 0;
}

int qb_last_fock_split(long long* quartets_fp64, long long* quartets_fp32)
{
    Context& c = ctx();
    if (int rc = fock_stats_resolve(c)) return rc;
    *quartets_fp32 = c.last_quartets32;
    *quartets_fp64 = c.last_quartets - c.last_quartets32;
    return 0;
}

int qb_last_fock_stats(long long* quartets, double* ms_eri, double* ms_screen)
{
    Context& c = ctx();
    if (int rc = fock_stats_resolve(c)) return rc;
    *quartets = c.last_quartets;
    *ms_eri = c.last_ms_eri;
    *ms_screen = c.last_ms_screen;
    return 0;
}

int qb_get_pairlist(int* xy, int cap, int* sorted_Q, int* sorted_Qnumber, int qcap, int* fStart, int* ffStart)
{
    Context& c = ctx();
    int n = (int)c.ref_xy.size() / 2;
    if (n > cap || c.Qshell > qcap) return -1;
    std::copy(c.ref_xy.begin(), c.ref_xy.end(), xy);
    std::copy(c.sorted_Q.begin(), c.sorted_Q.end(), sorted_Q);
    std::copy(c.sorted_Qnumber.begin(), c.sorted_Qnumber.end(), sorted_Qnumber);
    *fStart = c.fStart;
    *ffStart = c.ffStart;
    return n;
}

int qb_build_pairlist_host(int Qshell, const int* sorted_Q, const int* sorted_Qnumber, const int* kprim, int nshell,
                           const double* YCutoff, int* xy_out, int cap, int* fStart, int* ffStart)
{
    std::vector<int> xy;
    int n = build_pairlist(Qshell, sorted_Q, sorted_Qnumber, kprim, nshell, YCutoff, xy, *fStart, *ffStart);
    if (n > cap) return -1;
    std::copy(xy.begin(), xy.end(), xy_out);
    return n;
}

void gpu_cleanup_(void)
{
    if (!g) return;
    Context& c = *g;
    c.have_basis = c.have_pairs = c.have_calc = c.have_cutoff = false;
}

void gpu_upload_energy_(double* E)
{
    ctx().uploaded_energy = E ? *E : 0.0;
}

void gpu_upload_grad_(double* grad, double* gradCutoff)
{
    Context& c = ctx();
    c.grad_host.assign(grad, grad + 3 * (size_t)c.natom);
    c.gradCutoff = *gradCutoff;
    c.have_grad = true;
}

// grad <- grad + dE2/dR, E2 = sum (pq|rs) [D_pq D_rs / 2 - h D_pr D_qs / 4]
// (QUICK: gpu.cu:1481-1551 with getGrad_kernel, gpu_get2e_subs_grad.h).
void gpu_grad_(double* grad)
{
    Context& c = ctx();
    if (require(c.have_grad, "gpu_upload_grad_ must precede gpu_grad_")) return;
    if (require(c.have_calc, "gpu_upload_calculated_ must precede gpu_grad_")) return;
    size_t nn = (size_t)c.nbasis * c.nbasis;
    if (c.d_dense_raw.alloc(nn) != cudaSuccess ||
        cudaMemcpyAsync(c.d_dense_raw.p, c.d_dense_up.p, nn * sizeof(double), cudaMemcpyDeviceToDevice, c.stream) != cudaSuccess) {
        set_error(2, "copy of the density failed");
        return;
    }
    if (grad_build(c)) return;
    std::vector<double> g2(3 * (size_t)c.natom);
    if (cudaMemcpy(g2.data(), c.d_grad.p, g2.size() * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error(2, "download of the gradient failed");
        return;
    }
    for (size_t k = 0; k < g2.size(); k++) grad[k] = c.grad_host[k] + g2[k];
}
// Eelxc, aelec, belec <- input + grid sums; o <- symmetrised lower triangle
// of (O as uploaded + V_xc)  (QUICK: gpu.cu:1866-1975 with getxc_kernel).
void gpu_getxc_(int* isg, double* sigrad2, double* Eelxc, double* aelec, double* belec, double* o)
{
    Context& c = ctx();
    if (require(c.have_calc, "gpu_upload_calculated_ must precede gpu_getxc_")) return;
    if (require(c.have_basis && !c.xyz.empty(), "basis and coordinates must be uploaded before gpu_getxc_")) return;
    if (*isg != 1 && *isg != 2) {
        // QUICK's GPU path builds no grid points for SG0 (gridFormSG0 is
        // commented out, gpu_getxc.cu:117-121) and silently returns zeros.
        set_error(1, "gpu_getxc_: isg must be 1 (SG1) or 2 (75 x 302 Becke grid), got isg = %d", *isg);
        return;
    }
    const size_t nn = (size_t)c.nbasis * c.nbasis;
    if (c.d_dense_raw.alloc(nn) != cudaSuccess || c.d_o_out.alloc(nn) != cudaSuccess) {
        set_error(2, "cannot allocate %zu-element matrices", nn);
        return;
    }
    if (cudaMemcpyAsync(c.d_dense_raw.p, c.d_dense_up.p, nn * sizeof(double), cudaMemcpyDeviceToDevice, c.stream) != cudaSuccess ||
        cudaMemsetAsync(c.d_o_out.p, 0, nn * sizeof(double), c.stream) != cudaSuccess) {
        set_error(2, "upload of the density failed");
        return;
    }
    XcInputs in;
    in.natom = c.natom;
    in.nbasis = c.nbasis;
    in.maxcontract = c.maxcontract;
    in.method = c.method;
    in.xyz = c.xyz.data();
    in.iattype = c.iattype.data();
    in.ncenter = c.ncenter.data();
    in.itype = c.itype.data();
    in.ncontract = c.ncontract.data();
    in.aexp = c.aexp.data();
    in.dcoeff = c.dcoeff.data();
    in.sigrad2 = sigrad2;
    in.geom_version = c.geom_version;
    in.grid = *isg;
    in.stream = c.stream;
    XcResult r;
    if (xc_quadrature(in, c.d_dense_raw.p, c.d_o_out.p, &r)) return;
    c.last_xc = r;
    std::vector<double> v(nn);
    if (cudaMemcpyAsync(v.data(), c.d_o_out.p, nn * sizeof(double), cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
        cudaStreamSynchronize(c.stream) != cudaSuccess) {
        set_error(2, "download of V_xc failed");
        return;
    }
    const int n = c.nbasis;
    const std::vector<double>& oh = host_o(c);
    if (g_status) return;
    for (int i = 0; i < n; i++)
        for (int j = i; j < n; j++) {
            const size_t lo = (size_t)j + (size_t)i * n;   // (j, i), j >= i
            const double val = oh[lo] + v[lo];
            o[(size_t)i + (size_t)j * n] = val;
            o[lo] = val;
        }
    *Eelxc += r.exc;
    *aelec += r.nalpha;
    *belec += r.nalpha;
}
int gpu_schwarz_(double* YCutoff, double* cutPrim)
{
    Context& c = ctx();
    if (require(c.inited, "gpu_init_ must precede gpu_schwarz_")) return 1;
    if (require(c.have_basis && !c.xyz.empty(), "basis and coordinates must be uploaded before gpu_schwarz_")) return 1;
    struct Rec {
        int type, s1, s2, shA, LA, shB, LB;
        bool swapped;
    };
    std::vector<Rec> recs;
    for (int s1 = 0; s1 < c.nshell; s1++)
        for (int s2 = s1; s2 < c.nshell; s2++)
            for (int L1 = c.Qstart[s1]; L1 <= c.Qfinal[s1]; L1++)
                for (int L2 = c.Qstart[s2]; L2 <= c.Qfinal[s2]; L2++) {
                    Rec r{0, s1, s2, s1, L1, s2, L2, false};
                    if (L1 < L2) { r.shA = s2; r.LA = L2; r.shB = s1; r.LB = L1; r.swapped = true; }
                    r.type = pair_type_index(r.LA, r.LB);
                    if (r.type < 0) return set_error(1, "angular momentum (%d,%d) beyond this build", r.LA, r.LB), 1;
                    recs.push_back(r);
                }
    std::stable_sort(recs.begin(), recs.end(), [](const Rec& a, const Rec& b) { return a.type < b.type; });
    int nrec = (int)recs.size();
    std::vector<int4> pbf(nrec);
    std::vector<double4> pAB(nrec), prim;
    std::vector<int> tbeg(kNumPairTypes, 0), tend(kNumPairTypes, 0);
    for (int i = 0; i < nrec; i++) {
        const Rec& e = recs[i];
        const double *A = center(c, e.shA), *B = center(c, e.shB);
        double AB2 = 0;
        for (int k = 0; k < 3; k++) AB2 += (A[k] - B[k]) * (A[k] - B[k]);
        int off = (int)prim.size() / 3;
        for (int pa = 0; pa < c.kprim[e.shA]; pa++)
            for (int pb = 0; pb < c.kprim[e.shB]; pb++) {
                double a = cexpo(c, e.shA, pa), bb = cexpo(c, e.shB, pb), p = a + bb;
                double K = X0 * (exp(-a * bb / p * AB2) / p) * ccoef(c, e.shA, e.LA, pa) * ccoef(c, e.shB, e.LB, pb);
                double P[3], PA[3];
                for (int k = 0; k < 3; k++) {
                    P[k] = (A[k] * a + B[k] * bb) / p;
                    PA[k] = P[k] - A[k];
                }
                prim.push_back(make_double4(p, K, P[0], P[1]));
                prim.push_back(make_double4(P[2], PA[0], PA[1], PA[2]));
                prim.push_back(make_double4(0.5 / p, a, 0.0, 0.0));
            }
        pbf[i] = make_int4(bf_first(c, e.shA, e.LA), bf_first(c, e.shB, e.LB), off, (int)prim.size() / 3 - off);
        pAB[i] = make_double4(A[0] - B[0], A[1] - B[1], A[2] - B[2], 1.0);
        if (i == 0 || recs[i - 1].type != e.type) tbeg[e.type] = i;
        tend[e.type] = i + 1;
    }
    int nprimpair = (int)prim.size() / 3;
    CK(c.sw_prim.alloc(prim.size()));
    CK(c.sw_ab.alloc(nrec));
    CK(c.sw_bf.alloc(nrec));
    CK(c.sw_oc.alloc(nrec));
    CK(c.sw_op.alloc(nprimpair));
    CK(cudaMemcpyAsync(c.sw_prim.p, prim.data(), prim.size() * sizeof(double4), cudaMemcpyHostToDevice, c.stream));
    CK(cudaMemcpyAsync(c.sw_ab.p, pAB.data(), nrec * sizeof(double4), cudaMemcpyHostToDevice, c.stream));
    CK(cudaMemcpyAsync(c.sw_bf.p, pbf.data(), nrec * sizeof(int4), cudaMemcpyHostToDevice, c.stream));
    SchwarzParams S{c.sw_prim.p, c.sw_bf.p, c.sw_ab.p, c.d_cons.p, c.d_boys.p, c.sw_oc.p, c.sw_op.p};
    for (int t = 0; t < kNumPairTypes; t++) {
        if (tend[t] <= tbeg[t]) continue;
        int n = tend[t] - tbeg[t];
        int np = pbf[tend[t] - 1].z + pbf[tend[t] - 1].w - pbf[tbeg[t]].z;
        if (launch_schwarz(t, S, tbeg[t], tend[t], 0, std::min((n + 127) / 128, c.nsm * 8), 128, c.stream) < 0) {
            // pair types with an f shell: the generic recurrence program
            if (launch_generic_schwarz(kPairTypeL[t][0], kPairTypeL[t][1], S, tbeg[t], tend[t], 0, c.nsm, c.stream) < 0 ||
                launch_generic_schwarz(kPairTypeL[t][0], kPairTypeL[t][1], S, tbeg[t], tend[t], 1, c.nsm, c.stream) < 0)
                return set_error(5, "gpu_schwarz_: pair type (%d%d) needs more shared memory than this GPU offers",
                                 kPairTypeL[t][0], kPairTypeL[t][1]), 5;
            continue;
        }
        launch_schwarz(t, S, tbeg[t], tend[t], 1, std::min((np + 127) / 128, c.nsm * 8), 128, c.stream);
    }
    CK(cudaGetLastError());
    std::vector<double> oc(nrec), op(nprimpair);
    CK(cudaMemcpyAsync(oc.data(), c.sw_oc.p, nrec * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaMemcpyAsync(op.data(), c.sw_op.p, nprimpair * sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    int ns = c.nshell;
    std::vector<double> ymax((size_t)ns * ns, 0.0), pmax((size_t)c.jbasis * c.jbasis, 0.0);
    for (int i = 0; i < nrec; i++) {
        const Rec& e = recs[i];
        double& y = ymax[(size_t)e.s1 + (size_t)e.s2 * ns];
        y = std::max(y, oc[i]);
        int k = 0;
        for (int pa = 0; pa < c.kprim[e.shA]; pa++)
            for (int pb = 0; pb < c.kprim[e.shB]; pb++, k++) {
                int p1 = e.swapped ? pb : pa, p2 = e.swapped ? pa : pb;
                double& v = pmax[(size_t)(c.kstart[e.s1] - 1 + p1) + (size_t)(c.kstart[e.s2] - 1 + p2) * c.jbasis];
                v = std::max(v, op[pbf[i].z + k]);
            }
    }
    // cutPrim carries QUICK's extra factor X0 = 2 pi^2.5 (schwarz.f90:417)
    const double X0F = 2.0 * pow(3.1415926535897932384626433832795, 2.5);
    for (int s1 = 0; s1 < ns; s1++)
        for (int s2 = s1; s2 < ns; s2++) {
            double v = sqrt(ymax[(size_t)s1 + (size_t)s2 * ns]);
            YCutoff[(size_t)s1 + (size_t)s2 * ns] = v;
            YCutoff[(size_t)s2 + (size_t)s1 * ns] = v;
        }
    for (size_t k = 0; k < pmax.size(); k++) cutPrim[k] = sqrt(pmax[k] * X0F);
    return 0;
}

long long qb_launch_count(void) { return (long long)g_launches; }

int qb_fma_peak(int fp64, double* gflops)
{
    Context& c = ctx();
    if (require(c.inited, "gpu_init_ must precede qb_fma_peak")) return 1;
    return fma_probe(fp64, c.nsm, gflops, c.stream);
}

int qb_count_prim_quartets(long long* per_class, int cap)
{
    Context& c = ctx();
    if (require(c.have_pairs && c.d_quartets.p != nullptr, "a Fock build must precede qb_count_prim_quartets")) return 1;
    if (cap < kNumClasses) return set_error(1, "per_class needs %d entries", kNumClasses), 1;
    DevBuf<unsigned long long> d;
    CK(d.alloc(kNumClasses));
    CK(cudaMemsetAsync(d.p, 0, kNumClasses * sizeof(unsigned long long), c.stream));
    FockParams P = fock_params(c);
    launch_count_prims(P, kNumClasses, d.p, c.nsm, c.stream);
    CK(cudaGetLastError());
    std::vector<unsigned long long> h(kNumClasses);
    CK(cudaMemcpyAsync(h.data(), d.p, kNumClasses * sizeof(unsigned long long), cudaMemcpyDeviceToHost, c.stream));
    CK(cudaStreamSynchronize(c.stream));
    for (int k = 0; k < kNumClasses; k++) per_class[k] = (long long)h[k];
    return 0;
}

int qb_class_info(int* nclasses, int* class_L, long long* class_quartets, int cap)
{
    Context& c = ctx();
    *nclasses = kNumClasses;
    if (cap < kNumClasses) return 1;
    std::vector<int> cnt(kNumClasses, 0);
    if (c.d_class_count.p) CK(cudaMemcpy(cnt.data(), build_counts(c, 0), kNumClasses * sizeof(int), cudaMemcpyDeviceToHost));
    for (int k = 0; k < kNumClasses; k++) {
        for (int j = 0; j < 4; j++) class_L[4 * k + j] = kClassL[k][j];
        class_quartets[k] = cnt[k];
    }
    return 0;
}
// ------------------------------------------------- stored-integral path
// QUICK's conventional SCF (quick_method%nodirect, src/shell.f90:118-209 and
// src/cuda/gpu.cu:1559-2237): gpu_aoint_ computes every unique integral once
// and writes it to a file, gpu_addint_ reads the file each iteration and
// adds J and K for the uploaded density.  The file format is QUICK's: blocks
// of kEriBlock records, each block written as kEriBlock int IJ, then int KL,
// then double values (the last block short), IJ = i n + j, KL = k n + l.
constexpr int kEriBlock = 150000;   // BUFFERSIZE, gpu_common.h:44

// Fortran passes the name blank-padded: up to the first blank, like QUICK's trim()
static std::string fortran_name(const char* s)
{
    std::string r;
    for (int i = 0; i < 4096 && s[i] && s[i] != ' '; i++) r += s[i];
    return r;
}

__global__ void fill_kernel(double* p, size_t n, double v)
{
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) p[i] = v;
}

// Every distinct index permutation (p q|r s) of a stored integral adds
// D_rs Y to G_pq and -(h/2) D_qs Y to G_pr (the closed-shell two-electron
// operator summed over the permutations).
__global__ void addint_kernel(const EriRecord* __restrict__ rec, long long n, const double* __restrict__ D, int nb,
                              double hx, double* __restrict__ G)
{
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const EriRecord r = rec[t];
    const int i = r.IJ / nb, j = r.IJ % nb, k = r.KL / nb, l = r.KL % nb;
    const double y = r.value;
    const int P[8][4] = {{i, j, k, l}, {j, i, k, l}, {i, j, l, k}, {j, i, l, k},
                         {k, l, i, j}, {l, k, i, j}, {k, l, j, i}, {l, k, j, i}};
    for (int u = 0; u < 8; u++) {
        bool dup = false;
        for (int v = 0; v < u; v++)
            dup = dup || (P[u][0] == P[v][0] && P[u][1] == P[v][1] && P[u][2] == P[v][2] && P[u][3] == P[v][3]);
        if (dup) continue;
        const int p = P[u][0], q = P[u][1], rr = P[u][2], s = P[u][3];
        atomicAdd(G + p + (size_t)q * nb, __ldg(D + rr + (size_t)s * nb) * y);
        if (hx != 0.0) atomicAdd(G + p + (size_t)rr * nb, -0.5 * hx * __ldg(D + q + (size_t)s * nb) * y);
    }
}

// Shell quartets with Y_ij Y_kl > leastIntegralCutoff (QUICK's getAOInt
// screen: no density), integrals with |Y| > maxIntegralCutoff written;
// intNum += their number.  The class kernels store instead of digesting;
// classes are processed in slices that fit a 1 GB device record buffer.
void gpu_aoint_(double* leastIntegralCutoff, double* maxIntegralCutoff, int* intNum, char* intFileName)
{
    Context& c = ctx();
    if (require(c.have_pairs, "gpu_upload_cutoff_matrix_ must precede gpu_aoint_")) return;
    const std::string fname = fortran_name(intFileName);
    FILE* f = fopen(fname.c_str(), "wb");
    if (!f) {
        set_error(24, "gpu_aoint_: cannot open %s", fname.c_str());
        return;
    }
    const double saved_mixed = c.mixed_cut;
    c.integralCutoff = *leastIntegralCutoff;
    c.mixed_cut = 0.0;
    // a density screen of 1/4 everywhere makes DNMax = 1: the Schwarz test alone
    const size_t ns = c.nshell;
    if (c.d_cut_matrix.alloc(ns * ns) != cudaSuccess) { fclose(f); set_error(2, "gpu_aoint_: allocation failed"); return; }
    fill_kernel<<<(unsigned)((ns * ns + 255) / 256), 256, 0, c.stream>>>(c.d_cut_matrix.p, ns * ns, 0.25);
    ++g_launches;
    c.have_cutoff = true;
    auto fail = [&](const char* what) {
        fclose(f);
        c.mixed_cut = saved_mixed;
        c.have_cutoff = false;
        set_error(2, "gpu_aoint_: %s", what);
    };
    if ((g_sized_cutoff != c.integralCutoff || c.d_quartets.p == nullptr) && size_quartet_lists(c)) return fail("sizing");
    if (c.npass > 1) return fail("the quartet lists exceed the list memory budget (QB_LIST_BUDGET_MB); this path needs them whole");
    FockParams P = fock_params(c);
    ScreenParams S{c.d_screen_cls.p, c.d_counts.p, c.d_quartets.p, c.d_counts32.p};
    cudaMemsetAsync(c.d_counts.p, 0, kNumClasses * sizeof(unsigned long long), c.stream);
    cudaMemsetAsync(c.d_counts32.p, 0, kNumClasses * sizeof(unsigned long long), c.stream);
    cudaMemsetAsync(c.d_overflow.p, 0, sizeof(int), c.stream);
    launch_screen(S, P, kNumClasses, 0, c.nsm, c.stream);
    launch_finish_counts(S, c.d_class_count.p, c.d_class_count32.p, c.d_overflow.p, kNumClasses, c.stream);
    std::vector<int> cnt(kNumClasses);
    if (cudaMemcpyAsync(cnt.data(), c.d_class_count.p, kNumClasses * sizeof(int), cudaMemcpyDeviceToHost, c.stream) !=
            cudaSuccess || cudaStreamSynchronize(c.stream) != cudaSuccess)
        return fail("screen failed");
    const long long cap = 64LL << 20;   // records in the device buffer (1 GB)
    DevBuf<EriRecord> rec;
    DevBuf<unsigned long long> dcount;
    if (rec.alloc(cap) != cudaSuccess || dcount.alloc(1) != cudaSuccess) return fail("allocation failed");
    std::vector<int> A(kEriBlock), B(kEriBlock);
    std::vector<double> V(kEriBlock);
    std::vector<EriRecord> host;
    int nbuf = 0;
    long long total = 0;
    auto flush = [&](int m) {
        fwrite(A.data(), sizeof(int), m, f);
        fwrite(B.data(), sizeof(int), m, f);
        fwrite(V.data(), sizeof(double), m, f);
    };
    for (int k = 0; k < kNumClasses; k++) {
        if (cnt[k] == 0) continue;
        const int* Lk = kClassL[k];
        const long long ncomp = (long long)(Lk[0] + 1) * (Lk[0] + 2) / 2 * (Lk[1] + 1) * (Lk[1] + 2) / 2 *
                                (Lk[2] + 1) * (Lk[2] + 2) / 2 * (Lk[3] + 1) * (Lk[3] + 2) / 2;
        const long long slice = std::max(1LL, cap / ncomp);
        for (long long q0 = 0; q0 < cnt[k]; q0 += slice) {
            AoIntOut O{rec.p, dcount.p, cap, *maxIntegralCutoff, c.d_cons.p, c.nbasis, q0,
                       std::min<long long>(q0 + slice, cnt[k])};
            cudaMemsetAsync(dcount.p, 0, sizeof(unsigned long long), c.stream);
            const bool gen = kClassGeneric[k] || Lk[0] + Lk[1] + Lk[2] + Lk[3] >= c.generic_min_l;
            if (gen) {
                // the classes without straight-line kernels: the block-per-quartet store
                if (launch_generic_store(k, Lk[0], Lk[1], Lk[2], Lk[3], P, O, c.nsm, c.stream) < 0)
                    return fail("a class needs more shared memory than this GPU offers");
            } else {
                qb::g_aoint_out = &O;
                launch_class(k, P, -1, (int)(O.qend - O.qbegin), c.nsm, c.stream);
                qb::g_aoint_out = nullptr;
            }
            unsigned long long m = 0;
            if (cudaMemcpyAsync(&m, dcount.p, sizeof m, cudaMemcpyDeviceToHost, c.stream) != cudaSuccess ||
                cudaStreamSynchronize(c.stream) != cudaSuccess)
                return fail("kernel failed");
            if ((long long)m > cap) return fail("record buffer overflow (internal sizing error)");
            host.resize(m);
            if (m && cudaMemcpy(host.data(), rec.p, m * sizeof(EriRecord), cudaMemcpyDeviceToHost) != cudaSuccess)
                return fail("download failed");
            for (const EriRecord& r : host) {
                A[nbuf] = r.IJ;
                B[nbuf] = r.KL;
                V[nbuf] = r.value;
                if (++nbuf == kEriBlock) flush(nbuf), nbuf = 0;
            }
            total += (long long)m;
        }
    }
    flush(nbuf);
    fclose(f);
    c.mixed_cut = saved_mixed;
    c.have_cutoff = false;   // the density screen was replaced: the next build needs gpu_upload_cutoff_
    if (total > 2147483647LL) {
        set_error(25, "gpu_aoint_: %lld integrals exceed QUICK's int counter", total);
        return;
    }
    *intNum += (int)total;
}

// o <- symmetric (O as uploaded + J - (h/2) K) from the stored integrals of
// gpu_aoint_ and the density of the last gpu_upload_calculated_.
void gpu_addint_(double* o, int* intindex, char* intFileName)
{
    Context& c = ctx();
    if (require(c.have_calc, "gpu_upload_calculated_ must precede gpu_addint_")) return;
    const std::string fname = fortran_name(intFileName);
    FILE* f = fopen(fname.c_str(), "rb");
    if (!f) {
        set_error(24, "gpu_addint_: cannot open %s", fname.c_str());
        return;
    }
    const int n = c.nbasis;
    const size_t nn = (size_t)n * n;
    DevBuf<double> G;
    DevBuf<EriRecord> rec;
    if (G.alloc(nn) != cudaSuccess || rec.alloc(kEriBlock) != cudaSuccess || c.d_dense_raw.alloc(nn) != cudaSuccess) {
        fclose(f);
        set_error(2, "gpu_addint_: allocation failed");
        return;
    }
    cudaMemsetAsync(G.p, 0, nn * sizeof(double), c.stream);
    cudaMemcpyAsync(c.d_dense_raw.p, c.d_dense_up.p, nn * sizeof(double), cudaMemcpyDeviceToDevice, c.stream);
    const double hx = c.method == 0 ? 1.0 : (c.method == 1 ? 0.2 : 0.0);
    std::vector<int> A(kEriBlock), B(kEriBlock);
    std::vector<double> V(kEriBlock);
    std::vector<EriRecord> host(kEriBlock);
    long long remaining = *intindex;
    bool ok = true;
    while (remaining > 0 && ok) {
        const int m = (int)std::min<long long>(kEriBlock, remaining);
        ok = fread(A.data(), sizeof(int), m, f) == (size_t)m && fread(B.data(), sizeof(int), m, f) == (size_t)m &&
             fread(V.data(), sizeof(double), m, f) == (size_t)m;
        if (!ok) break;
        for (int i = 0; i < m; i++) host[i] = EriRecord{A[i], B[i], V[i]};
        ok = cudaMemcpyAsync(rec.p, host.data(), m * sizeof(EriRecord), cudaMemcpyHostToDevice, c.stream) == cudaSuccess;
        addint_kernel<<<(m + 255) / 256, 256, 0, c.stream>>>(rec.p, m, c.d_dense_raw.p, n, hx, G.p);
        ++g_launches;
        // the host buffers are refilled next: wait for this block's copy
        ok = ok && cudaStreamSynchronize(c.stream) == cudaSuccess;
        remaining -= m;
    }
    fclose(f);
    if (!ok) {
        set_error(24, "gpu_addint_: %s is shorter than %d records", fname.c_str(), *intindex);
        return;
    }
    std::vector<double> g(nn);
    if (cudaMemcpy(g.data(), G.p, nn * sizeof(double), cudaMemcpyDeviceToHost) != cudaSuccess) {
        set_error(2, "gpu_addint_: download failed");
        return;
    }
    const std::vector<double>& oh = host_o(c);
    if (g_status) return;
    for (size_t i = 0; i < nn; i++) o[i] = oh[i] + g[i];
}

}  // extern "C"

namespace qb {

// Read-only view of the current session's device tables, for entry points
// that bring their own working memory (noalloc.cu).  Working-memory fields of
// the returned FockParams (quartets, counts, dense, fock) are left null.
int session_view(SessionView* v)
{
    if (!g) return set_error(1, "no session: gpu_startup_ and the uploads must come first"), 1;
    Context& c = *g;
    if (require(c.inited, "gpu_init_ must come first")) return 1;
    if (require(c.have_pairs, "gpu_upload_cutoff_matrix_ must come first")) return 1;
    if (require(c.have_cutoff, "gpu_upload_cutoff_ must come first")) return 1;
    FockParams P = fock_params(c);
    P.quartets = nullptr;
    P.class_offset = nullptr;
    P.class_count = nullptr;
    P.dense = nullptr;
    P.fock = nullptr;
    v->P = P;
    v->cls = c.screen_cls;
    v->group = c.class_group;
    v->cons = c.d_cons.p;
    v->nsm = c.nsm;
    v->dev_id = c.dev_id;
    v->generic_min_l = c.generic_min_l;
    v->stream = c.stream;
    return 0;
}

int session_tables(const HostTables** t, FockParams* P, std::vector<int>* group, std::vector<int>* group32,
                   int* generic_min_l, int* nsm, int* method, double* mixed_cut)
{
    Context& c = ctx();
    if (require(c.have_pairs && c.have_basis, "a molecule's basis and pair list must be uploaded first")) return 1;
    *t = &c.host;
    *P = fock_params(c);
    *group = c.class_group;
    *group32 = c.class_group32;
    *generic_min_l = c.generic_min_l;
    *nsm = c.nsm;
    *method = c.method;
    *mixed_cut = c.mixed_cut;
    return 0;
}

int library_stream(cudaStream_t* st)
{
    Context& c = ctx();
    if (require(c.inited, "gpu_init_ must come first")) return 1;
    *st = c.stream;
    return 0;
}

int report_error(int code, const char* msg)
{
    set_error(code, "%s", msg);
    return code;
}

}  // namespace qb
