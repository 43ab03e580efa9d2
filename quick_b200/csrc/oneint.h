// Parameters of the one-electron integral and gradient kernels (oneint.cu).
#pragma once
#include <cuda_runtime.h>

namespace qb {

// One angular sub-shell of QUICK's basis (a shell's s, p, d or f part).
struct OneQ {
    int atom;      // 0-based centre
    int L;         // angular momentum
    int bf0;       // first basis function, 0-based
    int np;        // primitives
    int poff;      // offset of its primitives in pexp / pcoef
    int pad[3];
};

struct OneIntParams {
    const OneQ* q;
    const int2* pairs;          // (P, Q) sub-shell pairs, P <= Q, grouped by (L_P, L_Q)
    const double* xyz;          // (3, natom) bohr
    const double* chg;          // nuclear charges
    int natom, nbasis, maxcontract;
    int grad_shared;            // gradient: accumulate per block in shared memory
    const double* aexp;         // (maxcontract, nbasis)
    const double* dcoeff;       // (maxcontract, nbasis): per-function coefficients (S, T)
    const int* itype;           // (3, nbasis)
    const int* klmn;            // (3, nbasis)
    const double* cons;         // per-function factor of the V normalisation
    const double* pexp;         // primitive exponents per sub-shell
    const double* pcoef;        // gccoeff per sub-shell primitive (V)
    const double* boys;         // Boys table
    double* S;                  // outputs, nbasis x nbasis column-major (either may be null)
    double* H;
    const double* D;            // gradient inputs: total density and energy-weighted density
    const double* W;
    double* grad;               // (3, natom), accumulated
};

// Host description of the basis for oneint_run / grad1e_run (QUICK's arrays
// as gpu_upload_basis_ received them; Fortran layouts, 1-based stored indices).
struct OneIntHost {
    int natom, nbasis, nshell, maxcontract;
    const double* xyz;          // (3, natom) bohr
    const double* chg;
    const int *kprim, *katom, *Ksumtype, *Qstart, *Qfinal, *Qsbasis, *itype, *KLMN;
    const double *aexp, *dcoeff, *gccoeff, *gcexpo, *cons;
    const double* d_boys;       // device Boys table
    long long geom_version;     // changes whenever coordinates or basis change
    int nsm;
    cudaStream_t stream;
};

// S and H = T + V into device arrays (nbasis^2, column-major; either may be
// null), enqueued on h.stream.
int oneint_run(const OneIntHost& h, double* d_S, double* d_H);
// Adds the nuclear-repulsion and one-electron parts of the RHF gradient to
// d_grad (3 natom) from the total density D and energy-weighted density W
// (device, nbasis^2), enqueued on h.stream.
int grad1e_run(const OneIntHost& h, const double* d_D, const double* d_W, double* d_grad);

// Frees the device tables (session shutdown).
void oneint_release();

// Launch the S/H (grad = 0) or gradient (grad = 1) kernel of class (la, lb)
// over pairs[begin, end).  Returns -1 for an angular momentum above f.
int launch_oneint_class(int la, int lb, const OneIntParams& P, int begin, int end, int grad, int nsm, cudaStream_t st);
void launch_nuclear_grad(const OneIntParams& P, cudaStream_t st);

}  // namespace qb
