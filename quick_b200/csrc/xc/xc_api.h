// Host interface of the XC quadrature (xc.cu) used by the gpu_getxc_ bridge.
#pragma once
#include <cuda_runtime.h>

namespace qb {

struct XcInputs {
    int natom = 0, nbasis = 0, maxcontract = 0;
    int method = 1;                  // 1: B3LYP, 2: BLYP (QUICK's gpu_upload_method_ codes)
    const double* xyz = nullptr;     // (3, natom), bohr
    const int* iattype = nullptr;    // atomic numbers
    const int* ncenter = nullptr;    // (nbasis), 1-based atom of each basis function
    const int* itype = nullptr;      // (3, nbasis)
    const int* ncontract = nullptr;  // (nbasis)
    const double* aexp = nullptr;    // (maxcontract, nbasis)
    const double* dcoeff = nullptr;  // (maxcontract, nbasis), normalised
    const double* sigrad2 = nullptr; // (nbasis)
    long long geom_version = 0;      // changes whenever coordinates or basis change
    int grid = 1;                    // 1: QUICK's SG1 grid; 2: 75 x 302 grid with Becke's partition
    cudaStream_t stream = nullptr;
};

struct XcResult {
    double exc = 0.0;       // sum of w f over the grid
    double nalpha = 0.0;    // sum of w rho_alpha (QUICK's aelec; belec is the same)
    long long npts = 0;     // grid points kept (weight above the cutoff)
    long long nchunks = 0;  // point chunks with at least one significant basis function
    double ms = 0.0;        // device time of the per-call phase
    double ms_grid = 0.0;   // device time of the grid build (0 when cached)
    // algorithmic work of one call, summed over chunks of P points and nb
    // functions: bytes = P nb (phi, grad phi: 4 x 8 B) + 2 nb^2 x 8 B (D and
    // V tiles); flops = 4 P nb^2 (2 P nb^2 for rho, the same for V);
    // gemm_flops = what the two triangular products and the DGEMM
    // execute (P nb^2 + P nb^2 + 4 P nb^2).
    double alg_bytes = 0.0, alg_flops = 0.0, gemm_flops = 0.0;
};

// Accumulates V_xc into the lower triangle of d_v (column-major nbasis^2,
// V(j, i) for j >= i; the caller zeroes it) from the density d_dense
// (column-major nbasis^2).  Rebuilds the grid when geom_version or sigrad2
// changed.  Returns 0 or a QUICK-bridge status code after reporting the
// error.
int xc_quadrature(const XcInputs& in, const double* d_dense, double* d_v, XcResult* out);

// Adds the XC term of the nuclear gradient, dE_xc/dR (3 natom, the grid
// moving with the atoms, partition derivatives included), to d_grad for the
// density d_dense; ms: device time.  Synchronises the stream.
int xc_gradient(const XcInputs& in, const double* d_dense, double* d_grad, double* ms);

// Evaluates the functional (xc_functional.cuh) at n (rho, sigma) pairs on the
// device: out[3k] = f, out[3k+1] = df/drho, out[3k+2] = 4 df/dsigma.
int xc_functional_device(int method, int n, const double* d_rho, const double* d_sigma, double* d_out,
                         cudaStream_t st);

// Grid of the last build, for checking: copies up to cap points (x, y, z, w)
// in the order of the device arrays; returns the number of points.
long long xc_grid_points(double* xyzw, long long cap);

void xc_release();

}  // namespace qb
