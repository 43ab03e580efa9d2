// Internal declarations shared by the host bridge and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <vector>
#include "eri_common.cuh"
#include "grad_common.cuh"

namespace qb {

struct ScreenClass {
    int bra_begin, bra_end;     // bra pairs (indices into the pair table)
    int ket_begin, ket_end;     // ket pairs
    int same_type;              // bra and ket of the same pair type: kets b >= a only
    int seg_begin, seg_end;     // the ket type's constant primitive-count segments (FockParams::ket_segs)
    int counter;                // angular class: its counters and list region (a batch has one entry
                                // per molecule and class, all molecules' entries sharing the class's)
    long long out_offset;       // first slot of this class in the quartet buffer
    long long capacity;         // slots reserved for this class
};

// Host copies of one molecule's device tables (build_tables), for batches.
struct HostTables {
    int nbasis = 0, nshell = 0, natom = 0;
    std::vector<int4> pbf, psh;         // pair tables (FockParams::pair_bf, pair_sh)
    std::vector<double> pY;
    std::vector<double4> pAB, pA, prim;
    std::vector<PrimRec32> prim32;
    std::vector<int2> segs;             // constant primitive-count segments of each pair type
    std::vector<ScreenClass> scls;      // one per angular class
    std::vector<double> cons;           // per basis function
    std::vector<int> shell_atom;        // 0-based atom of each shell
    std::vector<int> shell_first;       // first basis function of each shell, nshell + 1 entries
};

struct ScreenParams {
    const ScreenClass* cls;
    unsigned long long* counts;     // FP64 quartets per class (from the front of the region)
    Quartet* out;
    unsigned long long* counts32;   // FP32 quartets per class (from the back), mixed precision only
};

struct SessionView {
    FockParams P;                       // session tables; working-memory pointers null
    std::vector<ScreenClass> cls;       // class ranges of the pair table
    std::vector<int> group;             // lanes per shell quartet of each class kernel
    const double* cons;
    int nsm;
    int dev_id;                         // the session's device
    int generic_min_l;                  // classes with L sum >= this run the generic kernel (as fock_build)
    cudaStream_t stream;
};
int session_view(SessionView* v);
// The current molecule's host tables and the session settings a batch needs.
int session_tables(const HostTables** t, FockParams* P, std::vector<int>* group, std::vector<int>* group32,
                   int* generic_min_l, int* nsm, int* method, double* mixed_cut);
// The library stream of an initialised session (qb_set_stream or its own).
int library_stream(cudaStream_t* st);
int report_error(int code, const char* msg);

// ncls screen entries (blockIdx.y); gx blocks per entry (0: 4 per SM)
void launch_screen(const ScreenParams& S, const FockParams& P, int ncls, int count_only, int nsm, cudaStream_t st,
                   int gx = 0);
void launch_finish_counts(const ScreenParams& S, int* class_count, int* class_count32, int* overflow, int ncls,
                          cudaStream_t st);
void launch_add_counts(const int* cnt, const int* cnt32, int* tot, int* tot32, int ncls, cudaStream_t st);
void launch_scale_density(const double* D, const double* cons, double* Ds, int n, cudaStream_t st);
void launch_fock_finish(const double* G, const double* cons, const double* Oin, double* Oout, int n, cudaStream_t st,
                        int fixed = 0);
// cut (nshell x nshell) = max |D| per shell-pair block; shell_first has nshell + 1 entries (0-based)
void launch_density_screen(const double* D, const int* shell_first, int nshell, int n, double* cut, cudaStream_t st);
void launch_add_vector(const double* x, double* y, int n, cudaStream_t st);
// Class kernels with G lanes per shell quartet (G not compiled for the
// class: 1); return the G launched.
int launch_class(int cls, const FockParams& P, int G, int nq, int nsm, cudaStream_t st);
int launch_class32(int cls, const FockParams& P, int G, int nq, int nsm, cudaStream_t st);
int class_max_group(int cls);
// launch codes of a class for the autotuner: lanes per quartet, and
// kSbFlag + lanes for the staged-Boys kernels of the light classes
int class_variants(int cls, int fp32, int* codes, int cap);
// The warp-per-quartet kernel of eri_generic.cu for any class (shells <= f);
// fp32_list: walk the class's FP32 list.  Returns -1 if the class needs more
// shared memory than the GPU offers.
struct AoIntOut;
int launch_generic_store(int cls, int la, int lb, int lc, int ld, const FockParams& P, const AoIntOut& O, int nsm,
                         cudaStream_t st);
int launch_generic_class(int cls, int la, int lb, int lc, int ld, const FockParams& P, int nq, int nsm, int fp32_list,
                         cudaStream_t st);
// Device bytes of the generic kernel's program of class (la lb|lc ld), and
// launch_generic_class with that program copied into caller memory (mem,
// 256-byte aligned, cap bytes) instead of memory of its own; -2 if cap is
// too small, -1 if the class needs more shared memory than the GPU offers.
size_t generic_program_bytes(int la, int lb, int lc, int ld);
int launch_generic_class_placed(int cls, int la, int lb, int lc, int ld, const FockParams& P, int nq, int nsm,
                                void* mem, size_t cap, cudaStream_t st);
// Forget the fixed-array addresses of qb_fock_device_static (session end).
void noalloc_reset();
// Free a many-molecule batch (batch.cu; session end).
void batch_release();
int launch_grad_class(int cls, const FockParams& P, const GradExtra& G, int GS, int nq, int nsm, cudaStream_t st);
// The FP32 gradient kernels of the mixed split, on the class's FP32 list; -1
// for a class without a straight-line gradient kernel.
int launch_grad_class32(int cls, const FockParams& P, const GradExtra& G, int GS, int nq, int nsm, cudaStream_t st);
// The gradient of a class with an f shell (eri_generic.cu); -1 if its scratch cannot be allocated.
int launch_generic_grad_class(int cls, int la, int lb, int lc, int ld, const FockParams& P, const GradExtra& X, int nq,
                              int nsm, int fp32_list, cudaStream_t st);
void generic_release();
int grad_max_group(int cls);
int session_grad_lanes(int k, int f32);   // the session's gradient lanes per quartet of class k
int fma_probe(int fp64, int nsm, double* gflops, cudaStream_t st);
void launch_count_prims(const FockParams& P, int ncls, unsigned long long* out, int nsm, cudaStream_t st);

}  // namespace qb
