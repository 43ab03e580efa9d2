/*
 * CPU oracle for the nuclear gradient of the two-electron energy.
 * TEST INFRASTRUCTURE ONLY (see oracle.c).
 *
 * E2 = sum_{pqrs} (pq|rs) [D_pq D_rs / 2 - h D_pr D_qs / 4], QUICK's RHF
 * convention with the total density D (src/gradient.f90:5-327 calls
 * getGrad_kernel, gpu_get2e_subs_grad.h:143-512, for this term).
 * Derivative integrals follow QUICK's construction: VRR to one higher
 * angular momentum, contraction weighted by 2 alpha / 2 beta / 2 gamma
 * (storeAA/BB/CC, gpu_get2e_subs_grad.h:318-350), HRR, and
 *   d/dA (ab|cd) = (a+1 b|cd)_{2a} - a_i (a-1 b|cd), likewise B, C;
 *   d/dD = -(d/dA + d/dB + d/dC)  (translational invariance, :499-501).
 * The same quartets as the Fock build are visited (QUICK's pair set, ii<=kk,
 * Schwarz and density screens, primitive screen, canonical integral filter);
 * quartets on a single atom are skipped as in QUICK (:89-92).  For each
 * canonical integral the density factor is summed over its distinct index
 * permutations, which is what QUICK's case table (:425-462) encodes.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* shared with oracle.c */
typedef struct {
    int natom, nbasis, nshell, jbasis;
    const double* xyz;
    const int *kstart, *katom, *kprim, *Ksumtype, *Qstart, *Qfinal, *Qsbasis, *Qfbasis, *KLMN;
    const double *gccoeff, *gcexpo, *cons;
} OBasis;

long oracle_shell_quartet_deriv(const OBasis* b, int ii, int jj, int kk, int ll, int I, int J, int K, int L,
                                double DNMax, const double* cutPrim, double primLimit, double* dA, double* dB,
                                double* dC);

static double perm_factor(const double* D, int n, int i, int j, int k, int l, double h)
{
    /* sum over the distinct images (pq|rs) of (ij|kl) of D_pq D_rs / 2 - h D_pr D_qs / 4 */
    int t[8][4] = {{i, j, k, l}, {j, i, k, l}, {i, j, l, k}, {j, i, l, k},
                   {k, l, i, j}, {l, k, i, j}, {k, l, j, i}, {l, k, j, i}};
    double s = 0.0;
    for (int a = 0; a < 8; a++) {
        int dup = 0;
        for (int c = 0; c < a && !dup; c++)
            if (t[c][0] == t[a][0] && t[c][1] == t[a][1] && t[c][2] == t[a][2] && t[c][3] == t[a][3]) dup = 1;
        if (dup) continue;
        int p = t[a][0], q = t[a][1], r = t[a][2], u = t[a][3];
        s += 0.5 * D[p + (size_t)q * n] * D[r + (size_t)u * n] - 0.25 * h * D[p + (size_t)r * n] * D[q + (size_t)u * n];
    }
    return s;
}

/* grad (3 natom) += dE2/dR.  Inputs as oracle_fock. */
void oracle_grad(const OBasis* b, const double* YCutoff, const double* cutPrim, const double* cutMatrix,
                 const double* dense, double integralCutoff, double primLimit, double hybrid, double* grad)
{
    int ns = b->nshell, nb = b->nbasis;
    /* Qshells sorted by angular momentum (gpu.cu:1191-1218) and QUICK's pair set */
    int nq = 0;
    for (int s = 0; s < ns; s++) nq += b->Qfinal[s] - b->Qstart[s] + 1;
    int *qs = malloc(sizeof(int) * nq), *qL = malloc(sizeof(int) * nq);
    int q = 0;
    for (int L = 0; L <= 3; L++)
        for (int s = 0; s < ns; s++)
            if (b->Qstart[s] <= L && L <= b->Qfinal[s]) { qs[q] = s; qL[q] = L; q++; }
    int* px = malloc(sizeof(int) * (size_t)nq * nq);
    int* py = malloc(sizeof(int) * (size_t)nq * nq);
    int np = 0;
    for (int x = 0; x < nq; x++)
        for (int y = 0; y < nq; y++)
            if (qs[x] <= qs[y] && YCutoff[qs[x] + (size_t)qs[y] * ns] > 1e-10) { px[np] = x; py[np] = y; np++; }
    double* gsum = calloc(3 * (size_t)b->natom, sizeof(double));
#pragma omp parallel
    {
        double* mine = calloc(3 * (size_t)b->natom, sizeof(double));
        size_t blk = 3 * 10 * 10 * 10 * 10;
        double *dA = malloc(sizeof(double) * blk), *dB = malloc(sizeof(double) * blk), *dC = malloc(sizeof(double) * blk);
#pragma omp for schedule(dynamic, 4)
        for (int a = 0; a < np; a++)
            for (int c = 0; c < np; c++) {
                int II = px[a], JJ = py[a], KK = px[c], LL = py[c];
                int ii = qs[II], jj = qs[JJ], kk = qs[KK], ll = qs[LL];
                if (ii > kk) continue;
                int at[4] = {b->katom[ii] - 1, b->katom[jj] - 1, b->katom[kk] - 1, b->katom[ll] - 1};
                if (at[0] == at[1] && at[0] == at[2] && at[0] == at[3]) continue;
#define CM(x, y) cutMatrix[(x) + (size_t)(y) * ns]
#define MX(x, y) ((x) >= (y) ? (x) : (y))
                double DNMax = MX(MX(4.0 * CM(ii, jj), 4.0 * CM(kk, ll)), MX(MX(CM(ii, ll), CM(ii, kk)), MX(CM(jj, kk), CM(jj, ll))));
                double yy = YCutoff[kk + (size_t)ll * ns] * YCutoff[ii + (size_t)jj * ns];
                if (!(yy > integralCutoff && yy * DNMax > integralCutoff)) continue;
                int I = qL[II], J = qL[JJ], K = qL[KK], L = qL[LL];
                oracle_shell_quartet_deriv(b, ii, jj, kk, ll, I, J, K, L, DNMax, cutPrim, primLimit, dA, dB, dC);
                int a0 = b->Ksumtype[ii] - 1 + b->Qsbasis[ii + (size_t)I * ns], a1 = b->Ksumtype[ii] - 1 + b->Qfbasis[ii + (size_t)I * ns];
                int b0 = b->Ksumtype[jj] - 1 + b->Qsbasis[jj + (size_t)J * ns], b1 = b->Ksumtype[jj] - 1 + b->Qfbasis[jj + (size_t)J * ns];
                int c0 = b->Ksumtype[kk] - 1 + b->Qsbasis[kk + (size_t)K * ns], c1 = b->Ksumtype[kk] - 1 + b->Qfbasis[kk + (size_t)K * ns];
                int d0 = b->Ksumtype[ll] - 1 + b->Qsbasis[ll + (size_t)L * ns], d1 = b->Ksumtype[ll] - 1 + b->Qfbasis[ll + (size_t)L * ns];
                int nJ = b1 - b0 + 1, nK = c1 - c0 + 1, nL = d1 - d0 + 1;
                for (int i = a0; i <= a1; i++)
                    for (int j = MX(i, b0); j <= b1; j++)
                        for (int k = MX(i, c0); k <= c1; k++)
                            for (int l = MX(k, d0); l <= d1; l++) {
                                if (!(i < k || (i == j && i == l) || (i == j && i < l) || (j == l && i < j) ||
                                      (i == k && i < j && j < l)))
                                    continue;
                                double g = perm_factor(dense, nb, i, j, k, l, hybrid);
                                size_t o = 3 * ((((size_t)(i - a0) * nJ + (j - b0)) * nK + (k - c0)) * nL + (l - d0));
                                for (int x = 0; x < 3; x++) {
                                    double ga = g * dA[o + x], gb = g * dB[o + x], gc = g * dC[o + x];
                                    mine[3 * at[0] + x] += ga;
                                    mine[3 * at[1] + x] += gb;
                                    mine[3 * at[2] + x] += gc;
                                    mine[3 * at[3] + x] -= ga + gb + gc;
                                }
                            }
            }
#pragma omp critical
        for (int k = 0; k < 3 * b->natom; k++) gsum[k] += mine[k];
        free(mine); free(dA); free(dB); free(dC);
    }
    for (int k = 0; k < 3 * b->natom; k++) grad[k] += gsum[k];
    free(gsum); free(qs); free(qL); free(px); free(py);
}
