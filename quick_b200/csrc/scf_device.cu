// Device pieces of the SCF iteration that the graph-captured SCF driver
// (quick_b200/scf.py, DeviceRHF.run with graph=True) cannot express as
// library GEMMs: the Pulay DIIS coefficients, solved on the device so the
// iteration never waits for the host (QUICK solves the same system on the
// host, src/scf.f90:249-523 with its LINEQ call).
#include <cuda_runtime.h>

#include "../../include/quick_b200.h"
#include "qb_internal.h"

namespace qb {

constexpr int kDiisMax = 32;

// Pulay's system over the m stored error vectors, slot i used when w[i] != 0:
//   sum_j B_ij c_j + lambda = 0 (used i),  sum_i c_i = 1,
// with the unused slots' rows and columns replaced by the identity (c_i = 0).
// Gaussian elimination with partial pivoting, one thread (m <= kDiisMax).  A
// singular system gives c = e_newest (no extrapolation), as QUICK's host
// falls back to the newest Fock matrix.
__global__ void diis_solve_kernel(const double* __restrict__ B, const double* __restrict__ w, int m,
                                  const long long* __restrict__ newest, double* __restrict__ c)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    constexpr int N = kDiisMax + 1;
    double A[N][N + 1];
    const int n = m + 1;
    for (int i = 0; i < m; i++) {
        const bool ui = w[i] != 0.0;
        for (int j = 0; j < m; j++) {
            const bool uj = w[j] != 0.0;
            A[i][j] = (ui && uj) ? B[i * m + j] : (i == j ? 1.0 : 0.0);
        }
        A[i][m] = ui ? 1.0 : 0.0;
        A[m][i] = ui ? 1.0 : 0.0;
        A[i][n] = 0.0;
    }
    A[m][m] = 0.0;
    A[m][n] = 1.0;
    bool ok = true;
    for (int k = 0; k < n && ok; k++) {
        int p = k;
        for (int i = k + 1; i < n; i++)
            if (fabs(A[i][k]) > fabs(A[p][k])) p = i;
        if (!(fabs(A[p][k]) > 0.0)) {
            ok = false;
            break;
        }
        if (p != k)
            for (int j = k; j <= n; j++) {
                const double t = A[k][j];
                A[k][j] = A[p][j];
                A[p][j] = t;
            }
        for (int i = k + 1; i < n; i++) {
            const double f = A[i][k] / A[k][k];
            for (int j = k; j <= n; j++) A[i][j] -= f * A[k][j];
        }
    }
    double x[N];
    for (int i = n - 1; i >= 0 && ok; i--) {
        double s = A[i][n];
        for (int j = i + 1; j < n; j++) s -= A[i][j] * x[j];
        x[i] = s / A[i][i];
        ok = ok && isfinite(x[i]);
    }
    const long long nw = *newest;
    for (int i = 0; i < m; i++) c[i] = ok ? x[i] : (i == nw ? 1.0 : 0.0);
}

}  // namespace qb

using namespace qb;

extern "C" int qb_diis_solve_device(const double* d_B, const double* d_w, int m, const long long* d_newest,
                                    double* d_c)
{
    if (m < 1 || m > kDiisMax) return report_error(1, "qb_diis_solve_device: m must be 1..32");
    cudaStream_t st = nullptr;
    if (int rc = library_stream(&st)) return rc;
    diis_solve_kernel<<<1, 32, 0, st>>>(d_B, d_w, m, d_newest, d_c);
    ++g_launches;
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return report_error(2, cudaGetErrorString(e));
    return 0;
}
