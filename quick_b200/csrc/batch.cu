// Many molecules in one Fock build or gradient (no counterpart in QUICK,
// which runs one molecule per process through gpu_get2e_).
//
// Each molecule is uploaded through the ordinary bridge (basis, Schwarz
// bounds, QUICK's pair list) and its tables are appended to the batch
// (qb_batch_add).  The batch concatenates the pair and primitive tables with
// global shell, pair and basis-function indices; its screen has one entry per
// (molecule, angular class), each pairing only bras and kets of its own
// molecule, and all molecules' quartets of a class go to that class's one
// list, so a build is one screen launch and one launch per class for the
// whole batch, whatever the number of molecules.  The class and gradient
// kernels are the single-molecule ones: they address the density and the
// Fock accumulator as one block-diagonal matrix of the batch's total
// dimension, of which only the diagonal blocks are ever written or read (the
// kernels here that scale the density, clear the accumulator, form the
// density screen and write the result visit only those blocks).  The caller
// passes and receives packed matrices: molecule i's n_i x n_i column-major
// block at offset off_i = sum_{j < i} n_j^2; gradients as 3 x natom_i blocks
// in molecule order.
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

#include "../../include/quick_b200.h"
#include "gen/eri_classes.h"
#include "qb_internal.h"

namespace qb {

namespace {

template <class T>
struct Buf {
    T* p = nullptr;
    size_t n = 0;
    cudaError_t alloc(size_t count)
    {
        if (count <= n && p) return cudaSuccess;
        release();
        n = count;
        return cudaMalloc((void**)&p, std::max<size_t>(count, 1) * sizeof(T));
    }
    cudaError_t upload(const std::vector<T>& v)
    {
        cudaError_t e = alloc(v.size());
        if (e != cudaSuccess || v.empty()) return e;
        return cudaMemcpy(p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
};

// per molecule: first basis function, dimension, packed offset; first shell, shells
struct MolInfo {
    int f0, n;
    long long pk;
    int s0, ns;
};

struct Batch {
    int nmol = 0, ntot = 0, nshtot = 0, natomtot = 0;
    long long pktot = 0;
    bool final = false;
    std::vector<MolInfo> mol;
    std::vector<int> natom;
    HostTables cat;                     // concatenated tables, global indices
    std::vector<ScreenClass> scls;      // nmol x ncls entries, molecule-major
    std::vector<int> shell_mol;
    double cutoff = 0.0, plim = 0.0;
    std::vector<long long> cap;         // per class: Schwarz-only quartet count
    Buf<double4> prim, pAB, pA;
    Buf<PrimRec32> prim32;
    Buf<int4> pbf, psh;
    Buf<double> pY, cons, dense, fock, cut;
    Buf<int2> segs;
    Buf<int> shell_atom, shell_first, dshell_mol;
    Buf<MolInfo> dmol;
    Buf<ScreenClass> dcls;
    Buf<unsigned long long> counts, counts32;
    Buf<int> ccount, ccount32, overflow;
    Buf<long long> coff, cend;
    Buf<Quartet> quartets;
    void release()
    {
        prim.release(); pAB.release(); pA.release(); prim32.release(); pbf.release(); psh.release();
        pY.release(); cons.release(); dense.release(); fock.release(); cut.release(); segs.release();
        shell_atom.release(); shell_first.release(); dshell_mol.release(); dmol.release(); dcls.release();
        counts.release(); counts32.release(); ccount.release(); ccount32.release(); overflow.release();
        coff.release(); cend.release(); quartets.release();
    }
};

Batch* g_batch = nullptr;

Batch& batch()
{
    if (!g_batch) g_batch = new Batch();
    return *g_batch;
}

#define BCK(call)                                                                                         \
    do {                                                                                                  \
        cudaError_t e_ = (call);                                                                          \
        if (e_ != cudaSuccess) return report_error(2, cudaGetErrorString(e_));                           \
    } while (0)

// ---------------------------------------------------------------- kernels
// blockIdx.y = molecule, threads over the n_i^2 elements of its block.

// D'(global a, b) = cons(a) cons(b) D_i(a, b) on the diagonal blocks
__global__ void batch_scale_density_kernel(const MolInfo* __restrict__ mol, const double* __restrict__ Dp,
                                           const double* __restrict__ cons, double* __restrict__ Ds, int ntot)
{
    const MolInfo m = mol[blockIdx.y];
    const long long nn = (long long)m.n * m.n;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(e % m.n), b = (int)(e / m.n);
        const int ga = m.f0 + a, gb = m.f0 + b;
        Ds[(size_t)gb * ntot + ga] = Dp[m.pk + e] * cons[ga] * cons[gb];
    }
}

// clear the diagonal blocks of the accumulator
__global__ void batch_zero_kernel(const MolInfo* __restrict__ mol, double* __restrict__ G, int ntot)
{
    const MolInfo m = mol[blockIdx.y];
    const long long nn = (long long)m.n * m.n;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(e % m.n), b = (int)(e / m.n);
        G[(size_t)(m.f0 + b) * ntot + (m.f0 + a)] = 0.0;
    }
}

// O_out,i(a, b) = O_in,i(a, b) + cons cons G(max, min), packed
__global__ void batch_finish_kernel(const MolInfo* __restrict__ mol, const double* __restrict__ G,
                                    const double* __restrict__ cons, const double* __restrict__ Oin,
                                    double* __restrict__ Oout, int ntot, int fixed)
{
    const MolInfo m = mol[blockIdx.y];
    const long long nn = (long long)m.n * m.n;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nn; e += (long long)gridDim.x * blockDim.x) {
        const int a = (int)(e % m.n), b = (int)(e / m.n);
        const int ga = m.f0 + a, gb = m.f0 + b;
        const int hi = ga > gb ? ga : gb, lo = ga > gb ? gb : ga;
        const size_t x = (size_t)hi * ntot + lo;
        const double g = fixed ? (double)reinterpret_cast<const long long*>(G)[x] / kFixedScale : G[x];
        Oout[m.pk + e] = Oin[m.pk + e] + cons[ga] * cons[gb] * g;
    }
}

// QUICK's density screen (schwarz.f90:550-600) per molecule: one block per
// global shell I, threads over the shells J >= I of its molecule.
__global__ void batch_density_screen_kernel(const MolInfo* __restrict__ mol, const int* __restrict__ shell_mol,
                                            const int* __restrict__ first, const double* __restrict__ Dp,
                                            int nshtot, double* __restrict__ cut)
{
    const int I = blockIdx.x;
    const MolInfo m = mol[shell_mol[I]];
    const int i0 = first[I] - m.f0, i1 = first[I + 1] - m.f0;
    for (int J = I + threadIdx.x; J < m.s0 + m.ns; J += blockDim.x) {
        const int j0 = first[J] - m.f0, j1 = first[J + 1] - m.f0;
        double v = 0.0;
        for (int j = j0; j < j1; j++)
            for (int i = i0; i < i1; i++) v = fmax(v, fabs(Dp[m.pk + i + (size_t)j * m.n]));
        cut[(size_t)I * nshtot + J] = v;
        cut[(size_t)J * nshtot + I] = v;
    }
}

dim3 block_grid(const Batch& B)
{
    long long maxnn = 1;
    for (const MolInfo& m : B.mol) maxnn = std::max(maxnn, (long long)m.n * m.n);
    return dim3((unsigned)std::min<long long>((maxnn + 255) / 256, 64), (unsigned)B.nmol);
}

FockParams batch_params(Batch& B, const FockParams& S)
{
    FockParams P = S;   // Boys tables, exchange fraction and mixed split from the session
    P.prim = B.prim.p;
    P.pair_bf = B.pbf.p;
    P.pair_sh = B.psh.p;
    P.pair_Y = B.pY.p;
    P.pair_AB = B.pAB.p;
    P.quartets = B.quartets.p;
    P.class_offset = B.coff.p;
    P.class_count = B.ccount.p;
    P.class_count32 = B.ccount32.p;
    P.class_end = B.cend.p;
    P.dense = B.dense.p;
    P.fock = B.fock.p;
    P.cut_matrix = B.cut.p;
    P.nbasis = B.ntot;
    P.nshell = B.nshtot;
    P.prim_limit = B.plim;
    P.integral_cutoff = B.cutoff;
    P.ket_segs = B.segs.p;
    P.prim32 = B.prim32.p;
    P.pair_A = B.pA.p;
    return P;
}

struct Session {
    const HostTables* t = nullptr;
    FockParams P;
    std::vector<int> g64, g32;
    int generic_min_l = 99, nsm = 148, method = 0;
    double mixed_cut = 0.0;
    cudaStream_t st = nullptr;
};

int get_session(Session& s)
{
    if (int rc = session_tables(&s.t, &s.P, &s.g64, &s.g32, &s.generic_min_l, &s.nsm, &s.method, &s.mixed_cut))
        return rc;
    return library_stream(&s.st);
}

int need_final(const Batch& B)
{
    if (!B.final) return report_error(1, "qb_batch_finalize must precede the batched builds");
    return 0;
}

// density screen and scaled density of the packed D, then the screen into the class lists
int batch_screen(Batch& B, const FockParams& P, const double* d_dense, int nsm, cudaStream_t st)
{
    BCK(cudaMemsetAsync(B.counts.p, 0, kNumClasses * sizeof(unsigned long long), st));
    BCK(cudaMemsetAsync(B.counts32.p, 0, kNumClasses * sizeof(unsigned long long), st));
    BCK(cudaMemsetAsync(B.overflow.p, 0, sizeof(int), st));
    batch_density_screen_kernel<<<B.nshtot, 64, 0, st>>>(B.dmol.p, B.dshell_mol.p, B.shell_first.p, d_dense, B.nshtot,
                                                         B.cut.p);
    batch_scale_density_kernel<<<block_grid(B), 256, 0, st>>>(B.dmol.p, d_dense, B.cons.p, B.dense.p, B.ntot);
    g_launches += 2;
    ScreenParams S{B.dcls.p, B.counts.p, B.quartets.p, B.counts32.p};
    launch_screen(S, P, (int)B.scls.size(), 0, nsm, st, 2);
    launch_finish_counts(S, B.ccount.p, B.ccount32.p, B.overflow.p, kNumClasses, st);
    BCK(cudaGetLastError());
    return 0;
}

}  // namespace
}  // namespace qb

using namespace qb;

void qb::batch_release()
{
    if (g_batch) {
        g_batch->release();
        delete g_batch;
        g_batch = nullptr;
    }
}

extern "C" int qb_batch_reset(void)
{
    batch_release();
    return 0;
}

extern "C" int qb_batch_add(void)
{
    Batch& B = batch();
    if (B.final) return report_error(1, "qb_batch_add: the batch is finalized (qb_batch_reset starts a new one)");
    Session s;
    if (int rc = get_session(s)) return rc;
    const HostTables& t = *s.t;
    const int po = (int)B.cat.pbf.size(), qo = (int)B.cat.prim32.size(), so = (int)B.cat.segs.size();
    MolInfo m{B.ntot, t.nbasis, B.pktot, B.nshtot, t.nshell};
    for (int4 v : t.pbf) B.cat.pbf.push_back(make_int4(v.x + m.f0, v.y + m.f0, v.z + qo, v.w));
    for (int4 v : t.psh) B.cat.psh.push_back(make_int4(v.x + m.s0, v.y + m.s0, v.z + 4 * m.s0, v.w));
    B.cat.pY.insert(B.cat.pY.end(), t.pY.begin(), t.pY.end());
    B.cat.pAB.insert(B.cat.pAB.end(), t.pAB.begin(), t.pAB.end());
    B.cat.pA.insert(B.cat.pA.end(), t.pA.begin(), t.pA.end());
    B.cat.prim.insert(B.cat.prim.end(), t.prim.begin(), t.prim.end());
    B.cat.prim32.insert(B.cat.prim32.end(), t.prim32.begin(), t.prim32.end());
    for (int2 v : t.segs) B.cat.segs.push_back(make_int2(v.x + po, v.y + po));
    for (const ScreenClass& c : t.scls) {
        ScreenClass e = c;
        e.bra_begin += po; e.bra_end += po; e.ket_begin += po; e.ket_end += po;
        e.seg_begin += so; e.seg_end += so;
        e.out_offset = 0;
        e.capacity = 0;
        B.scls.push_back(e);
    }
    B.cat.cons.insert(B.cat.cons.end(), t.cons.begin(), t.cons.end());
    for (int a : t.shell_atom) B.cat.shell_atom.push_back(a + B.natomtot);
    for (int sh = 0; sh < t.nshell; sh++) {
        B.cat.shell_first.push_back(t.shell_first[sh] + m.f0);
        B.shell_mol.push_back(B.nmol);
    }
    B.mol.push_back(m);
    B.natom.push_back(t.natom);
    B.ntot += t.nbasis;
    B.nshtot += t.nshell;
    B.natomtot += t.natom;
    B.pktot += (long long)t.nbasis * t.nbasis;
    B.nmol++;
    return 0;
}

extern "C" int qb_batch_finalize(double integralCutoff, double primLimit)
{
    Batch& B = batch();
    if (B.nmol == 0) return report_error(1, "qb_batch_finalize: no molecules added");
    if ((long long)B.nmol * kNumClasses > 65535)
        return report_error(1, "qb_batch_finalize: at most 65535 / (angular classes) molecules per batch");
    if (B.final) return report_error(1, "qb_batch_finalize: already finalized");
    Session s;
    if (int rc = get_session(s)) return rc;
    B.cutoff = integralCutoff;
    B.plim = primLimit;
    B.cat.shell_first.push_back(B.ntot);
    // block-diagonal work matrices of the total dimension (only the blocks are touched)
    const double gb = ((double)B.ntot * B.ntot * 2.0 + (double)B.nshtot * B.nshtot) * 8.0 / 1e9;
    if (gb > 120.0) return report_error(1, "qb_batch_finalize: the batch's work matrices exceed 120 GB");
    BCK(B.prim.upload(B.cat.prim));
    BCK(B.prim32.upload(B.cat.prim32));
    BCK(B.pbf.upload(B.cat.pbf));
    BCK(B.psh.upload(B.cat.psh));
    BCK(B.pY.upload(B.cat.pY));
    BCK(B.pAB.upload(B.cat.pAB));
    BCK(B.pA.upload(B.cat.pA));
    BCK(B.segs.upload(B.cat.segs));
    BCK(B.cons.upload(B.cat.cons));
    BCK(B.shell_atom.upload(B.cat.shell_atom));
    BCK(B.shell_first.upload(B.cat.shell_first));
    BCK(B.dshell_mol.upload(B.shell_mol));
    BCK(B.dmol.upload(B.mol));
    BCK(B.dense.alloc((size_t)B.ntot * B.ntot));
    BCK(B.fock.alloc((size_t)B.ntot * B.ntot));
    BCK(B.cut.alloc((size_t)B.nshtot * B.nshtot));
    BCK(B.counts.alloc(kNumClasses));
    BCK(B.counts32.alloc(kNumClasses));
    BCK(B.ccount.alloc(kNumClasses));
    BCK(B.ccount32.alloc(kNumClasses));
    BCK(B.overflow.alloc(1));
    BCK(B.coff.alloc(kNumClasses));
    BCK(B.cend.alloc(kNumClasses));
    // Schwarz-only counts size each class's list (an upper bound for every density)
    BCK(B.dcls.upload(B.scls));
    BCK(cudaMemset(B.counts.p, 0, kNumClasses * sizeof(unsigned long long)));
    FockParams P = batch_params(B, s.P);
    ScreenParams S{B.dcls.p, B.counts.p, nullptr, B.counts32.p};
    launch_screen(S, P, (int)B.scls.size(), 1, s.nsm, s.st, 2);
    BCK(cudaGetLastError());
    std::vector<unsigned long long> cnt(kNumClasses);
    BCK(cudaMemcpyAsync(cnt.data(), B.counts.p, kNumClasses * sizeof(unsigned long long), cudaMemcpyDeviceToHost, s.st));
    BCK(cudaStreamSynchronize(s.st));
    B.cap.assign(kNumClasses, 0);
    std::vector<long long> offs(kNumClasses), ends(kNumClasses);
    long long off = 0;
    for (int k = 0; k < kNumClasses; k++) {
        B.cap[k] = (long long)cnt[k];
        offs[k] = off;
        off += B.cap[k];
        ends[k] = off;
    }
    for (ScreenClass& e : B.scls) {
        e.out_offset = offs[e.counter];
        e.capacity = B.cap[e.counter];
    }
    BCK(B.dcls.upload(B.scls));
    BCK(B.quartets.alloc((size_t)std::max<long long>(off, 1)));
    BCK(cudaMemcpy(B.coff.p, offs.data(), kNumClasses * sizeof(long long), cudaMemcpyHostToDevice));
    BCK(cudaMemcpy(B.cend.p, ends.data(), kNumClasses * sizeof(long long), cudaMemcpyHostToDevice));
    B.final = true;
    return 0;
}

extern "C" int qb_batch_layout(int* nbasis, int* natom, long long* offsets, int cap)
{
    Batch& B = batch();
    for (int i = 0; i < std::min(cap, B.nmol); i++) {
        nbasis[i] = B.mol[i].n;
        natom[i] = B.natom[i];
        offsets[i] = B.mol[i].pk;
    }
    return B.nmol;
}

extern "C" int qb_batch_fock_device(const double* d_dense, const double* d_o_in, double* d_o_out)
{
    Batch& B = batch();
    if (int rc = need_final(B)) return rc;
    Session s;
    if (int rc = get_session(s)) return rc;
    FockParams P = batch_params(B, s.P);
    batch_zero_kernel<<<block_grid(B), 256, 0, s.st>>>(B.dmol.p, B.fock.p, B.ntot);
    ++g_launches;
    if (int rc = batch_screen(B, P, d_dense, s.nsm, s.st)) return rc;
    for (int k = 0; k < kNumClasses; k++) {
        if (B.cap[k] == 0) continue;
        const int nq = (int)std::min<long long>(B.cap[k], 1LL << 30);
        const int* Lk = kClassL[k];
        const bool gen = Lk[0] + Lk[1] + Lk[2] + Lk[3] >= s.generic_min_l;
        for (int f32 = 0; f32 < (s.mixed_cut > 0.0 ? 2 : 1); f32++) {
            const int G = f32 ? (s.g32.empty() ? 1 : s.g32[k]) : (s.g64.empty() ? 1 : s.g64[k]);
            const int rc = gen ? launch_generic_class(k, Lk[0], Lk[1], Lk[2], Lk[3], P, nq, s.nsm, f32, s.st)
                               : (f32 ? launch_class32(k, P, G, nq, s.nsm, s.st) : launch_class(k, P, G, nq, s.nsm, s.st));
            if (rc < 0) return report_error(5, "qb_batch_fock_device: a class needs more shared memory than the GPU offers");
        }
    }
    batch_finish_kernel<<<block_grid(B), 256, 0, s.st>>>(B.dmol.p, B.fock.p, B.cons.p, d_o_in, d_o_out, B.ntot,
                                                          P.fixed_point);
    ++g_launches;
    BCK(cudaGetLastError());
    return 0;
}

extern "C" int qb_batch_grad_device(const double* d_dense, double* d_grad)
{
    Batch& B = batch();
    if (int rc = need_final(B)) return rc;
    Session s;
    if (int rc = get_session(s)) return rc;
    FockParams P = batch_params(B, s.P);
    if (int rc = batch_screen(B, P, d_dense, s.nsm, s.st)) return rc;
    GradExtra GX{B.shell_atom.p, B.psh.p, d_grad, B.natomtot, 3 * B.natomtot * 8 <= 48 * 1024 ? 1 : 0};
    for (int k = 0; k < kNumClasses; k++) {
        if (B.cap[k] == 0) continue;
        const int nq = (int)std::min<long long>(B.cap[k], 1LL << 30);
        for (int f32 = 0; f32 < (s.mixed_cut > 0.0 ? 2 : 1); f32++) {
            const int GS = session_grad_lanes(k, f32);
            const int rc = f32 ? launch_grad_class32(k, P, GX, GS, nq, s.nsm, s.st)
                               : launch_grad_class(k, P, GX, GS, nq, s.nsm, s.st);
            if (rc < 0) {
                const int* Lk = kClassL[k];
                if (launch_generic_grad_class(k, Lk[0], Lk[1], Lk[2], Lk[3], P, GX, nq, s.nsm, f32, s.st) < 0)
                    return report_error(2, "qb_batch_grad_device: cannot allocate the scratch of an f-shell class");
            }
        }
    }
    BCK(cudaGetLastError());
    return 0;
}
