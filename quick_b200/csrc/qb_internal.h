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
    long long out_offset;       // first slot of this class in the quartet buffer
    long long capacity;         // slots reserved for this class
};

struct ScreenParams {
    const ScreenClass* cls;
    unsigned long long* counts;
    int2* out;
};

struct SessionView {
    FockParams P;                       // session tables; working-memory pointers null
    std::vector<ScreenClass> cls;       // class ranges of the pair table
    const double* cons;
    int nsm;
    cudaStream_t stream;
};
int session_view(SessionView* v);
int report_error(int code, const char* msg);

void launch_screen(const ScreenParams& S, const FockParams& P, int ncls, int count_only, int nsm, cudaStream_t st);
void launch_finish_counts(const ScreenParams& S, int* class_count, int* overflow, int ncls, cudaStream_t st);
void launch_scale_density(const double* D, const double* cons, double* Ds, int n, cudaStream_t st);
void launch_fock_finish(const double* G, const double* cons, const double* Oin, double* Oout, int n, cudaStream_t st);
void launch_class(int cls, const FockParams& P, int grid, int block, cudaStream_t st);
void launch_grad_class(int cls, const FockParams& P, const GradExtra& G, int grid, int block, cudaStream_t st);
int fma_probe(int fp64, int nsm, double* gflops, cudaStream_t st);
void launch_count_prims(const FockParams& P, int ncls, unsigned long long* out, int nsm, cudaStream_t st);

}  // namespace qb
