/*
 * CPU oracle for the direct-SCF two-electron path of QUICK.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's cpu_baseline leg may load this file's library, and only as the
 * checker.  The product (quick_b200) never calls it.
 *
 * A plain-C restatement of the reference's algorithm, written for clarity
 * rather than speed:
 *   - Boys function F_m(T) evaluated to full double precision (series in
 *     long double below T=35, asymptotic + upward recursion above);
 *   - Head-Gordon-Pople / Obara-Saika vertical recurrence [e0|f0]^(m)
 *     (gpu_get2e_subs.h:586-747 drives int.h:714 `vertical`), contracted over
 *     primitives, then horizontal recurrence to (ab|cd)
 *     (gpu_get2e_subs_hrr.h:16-60), scaled by cons() per component;
 *   - Schwarz bounds YCutoff / cutPrim exactly as schwarz.f90:12-548 defines
 *     them (including cutPrim's extra factor X0 = 2 pi^2.5, classprim:417);
 *   - density screen cutMatrix (schwarz.f90:550-599);
 *   - the Fock build of get2e_kernel (gpu_get2e_subs.h:75-407): the same
 *     shell-pair set, the same ii<=kk rule, the same quartet and primitive
 *     screens evaluated in the same floating-point order, the same canonical
 *     basis-function filter (gpu_get2e_subs.h:792-801) and addint's six
 *     scatters (gpu_get2e_subs.h:1296-1384), accumulated in double.
 * Parity is pinned against QUICK's own bridge and kernels compiled as host
 * code (oracle/_ref) and against QUICK's published HF energies.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define MAXL 3                 /* f shells */
#define MAXLSUM (4 * MAXL + 2) /* bra+ket total angular momentum (+2 for gradient) */
#define NCART(n) (((n) + 1) * ((n) + 2) / 2)
#define MAXPRIM 10

static const double PI_ = 3.1415926535897932384626433832795;

/* ---------------------------------------------------------------- Boys */
/* F_m(T) for m = 0..mmax.  Series F_m(T) = e^{-T} sum_k (2T)^k / ((2m+1)(2m+3)...(2m+2k+1))
 * for T < 35 (evaluated for m = mmax in long double, then downward
 * recursion F_{m} = (2T F_{m+1} + e^{-T})/(2m+1), which is stable);
 * for T >= 35 the asymptotic F_0 = sqrt(pi/T)/2 plus upward recursion, whose
 * relative error there is below 1e-15 up to m = 16. */
void oracle_boys(int mmax, double T, double* F)
{
    if (T < 35.0) {
        long double t = T, e = expl(-t);
        long double term = 1.0L / (2 * mmax + 1), sum = term;
        for (int k = 1; k < 400; k++) {
            term *= 2.0L * t / (2 * mmax + 2 * k + 1);
            sum += term;
            if (term < sum * 1e-21L) break;
        }
        long double f = e * sum;
        F[mmax] = (double)f;
        for (int m = mmax - 1; m >= 0; m--) {
            f = (2.0L * t * f + e) / (2 * m + 1);
            F[m] = (double)f;
        }
    } else {
        long double t = T, e = expl(-t);
        long double f = 0.5L * sqrtl((long double)PI_ / t);
        F[0] = (double)f;
        for (int m = 1; m <= mmax; m++) {
            f = ((2 * m - 1) * f - e) / (2.0L * t);
            F[m] = (double)f;
        }
    }
}

/* ------------------------------------------------- Cartesian indexing */
/* Global index of a Cartesian exponent triple over all shells of total
 * angular momentum <= MAXLSUM: offset(n) + position inside shell n. */
static int cart_index[MAXLSUM + 2][MAXLSUM + 2][MAXLSUM + 2];
static int cart_xyz[4096][3];
static int cart_ready = 0;

static void cart_init(void)
{
    if (cart_ready) return;
    int idx = 0;
    for (int n = 0; n <= MAXLSUM + 1; n++)
        for (int x = n; x >= 0; x--)
            for (int y = n - x; y >= 0; y--) {
                int z = n - x - y;
                cart_index[x][y][z] = idx;
                cart_xyz[idx][0] = x;
                cart_xyz[idx][1] = y;
                cart_xyz[idx][2] = z;
                idx++;
            }
    cart_ready = 1;
}
static inline int cidx(int x, int y, int z) { return cart_index[x][y][z]; }
static inline int ncart_upto(int n) { return (n + 1) * (n + 2) * (n + 3) / 6; } /* shells 0..n */

/* ------------------------------------------------------------- basis */
typedef struct {
    int natom, nbasis, nshell, jbasis;
    const double* xyz;                 /* (3, natom) bohr */
    const int *kstart, *katom, *kprim, *Ksumtype, *Qstart, *Qfinal, *Qsbasis, *Qfbasis, *KLMN;
    const double *gccoeff, *gcexpo, *cons;
} OBasis;

#define F2(A, i, j, d1) (A)[(i) + (size_t)(j) * (d1)]

static inline const double* center(const OBasis* b, int shell)
{
    return b->xyz + 3 * (b->katom[shell] - 1);
}
/* first / last basis function (0-based) of sub-shell (shell, L) */
static inline int bf_first(const OBasis* b, int sh, int L) { return b->Ksumtype[sh] - 1 + F2(b->Qsbasis, sh, L, b->nshell); }
static inline int bf_last(const OBasis* b, int sh, int L) { return b->Ksumtype[sh] - 1 + F2(b->Qfbasis, sh, L, b->nshell); }
/* contraction coefficient of primitive p of sub-shell (sh, L): QUICK uses
 * the coefficient stored for component Ksumtype(sh)+L (shell.f90:74-76,
 * gpu.cu:1290-1300) */
static inline double ccoef(const OBasis* b, int sh, int L, int p) { return F2(b->gccoeff, p, b->Ksumtype[sh] - 1 + L, MAXPRIM); }
static inline double cexpo(const OBasis* b, int sh, int p) { return F2(b->gcexpo, p, b->Ksumtype[sh] - 1, MAXPRIM); }

/* ------------------------------------------------ primitive-quartet VRR */
/* Work space for [e0|f0]^(m):  A[(ie * nf + jf) * (M+1) + m] */
typedef struct {
    int Lab, Lcd, M;
    int ne, nf;         /* number of Cartesian triples with |e|<=Lab, |f|<=Lcd */
    double* A;
} VrrWork;

static void vrr_alloc(VrrWork* w, int Lab, int Lcd)
{
    w->Lab = Lab; w->Lcd = Lcd; w->M = Lab + Lcd;
    w->ne = ncart_upto(Lab); w->nf = ncart_upto(Lcd);
    w->A = (double*)malloc(sizeof(double) * (size_t)w->ne * w->nf * (w->M + 1));
}
#define VA(w, ie, jf, m) (w)->A[((size_t)(ie) * (w)->nf + (jf)) * ((w)->M + 1) + (m)]

/* One primitive quartet: fills [e0|f0]^(m) for all |e|<=Lab, |f|<=Lcd. */
static void vrr_prim(VrrWork* w, const double* A, const double* C, double a, double bexp,
                     double c, double d, const double* Bc, const double* Dc, double pref)
{
    double p = a + bexp, q = c + d, pq = p + q;
    double P[3], Q[3], W[3], PA[3], QC[3], WP[3], WQ[3];
    double rho = p * q / pq, T = 0.0;
    for (int i = 0; i < 3; i++) {
        P[i] = (a * A[i] + bexp * Bc[i]) / p;
        Q[i] = (c * C[i] + d * Dc[i]) / q;
        W[i] = (p * P[i] + q * Q[i]) / pq;
        PA[i] = P[i] - A[i];
        QC[i] = Q[i] - C[i];
        WP[i] = W[i] - P[i];
        WQ[i] = W[i] - Q[i];
        T += (P[i] - Q[i]) * (P[i] - Q[i]);
    }
    T *= rho;
    double F[MAXLSUM + 4];
    int M = w->M;
    oracle_boys(M, T, F);
    for (int m = 0; m <= M; m++) VA(w, 0, 0, m) = pref * F[m];
    double o2p = 0.5 / p, o2q = 0.5 / q, o2pq = 0.5 / pq, rp = rho / p, rq = rho / q;
    /* bra: [e0|00]^(m) */
    for (int n = 1; n <= w->Lab; n++)
        for (int ie = ncart_upto(n - 1); ie < ncart_upto(n); ie++) {
            int e[3] = {cart_xyz[ie][0], cart_xyz[ie][1], cart_xyz[ie][2]};
            int i = e[0] ? 0 : (e[1] ? 1 : 2);
            e[i]--;
            int e1 = cidx(e[0], e[1], e[2]);
            int e2 = -1;
            double ni = e[i];
            if (e[i] > 0) { e[i]--; e2 = cidx(e[0], e[1], e[2]); }
            for (int m = 0; m <= M - n; m++) {
                double v = PA[i] * VA(w, e1, 0, m) + WP[i] * VA(w, e1, 0, m + 1);
                if (e2 >= 0) v += ni * o2p * (VA(w, e2, 0, m) - rp * VA(w, e2, 0, m + 1));
                VA(w, ie, 0, m) = v;
            }
        }
    /* ket: [e0|f0]^(m) */
    for (int n = 1; n <= w->Lcd; n++)
        for (int jf = ncart_upto(n - 1); jf < ncart_upto(n); jf++) {
            int f[3] = {cart_xyz[jf][0], cart_xyz[jf][1], cart_xyz[jf][2]};
            int i = f[0] ? 0 : (f[1] ? 1 : 2);
            f[i]--;
            int f1 = cidx(f[0], f[1], f[2]);
            int f2 = -1;
            double ni = f[i];
            if (f[i] > 0) { f[i]--; f2 = cidx(f[0], f[1], f[2]); }
            for (int ie = 0; ie < ncart_upto(w->Lab); ie++) {
                int ne_ = cart_xyz[ie][0] + cart_xyz[ie][1] + cart_xyz[ie][2];
                int ei = cart_xyz[ie][i];
                int em = -1;
                if (ei > 0) {
                    int e[3] = {cart_xyz[ie][0], cart_xyz[ie][1], cart_xyz[ie][2]};
                    e[i]--;
                    em = cidx(e[0], e[1], e[2]);
                }
                for (int m = 0; m <= M - n - ne_; m++) {
                    double v = QC[i] * VA(w, ie, f1, m) + WQ[i] * VA(w, ie, f1, m + 1);
                    if (f2 >= 0) v += ni * o2q * (VA(w, ie, f2, m) - rq * VA(w, ie, f2, m + 1));
                    if (em >= 0) v += ei * o2pq * VA(w, em, f1, m + 1);
                    VA(w, ie, jf, m) = v;
                }
            }
        }
}

/* -------------------------------------------------------------- HRR */
/* G[ie * nfull + jf] holds contracted (e0|f0); ket-side and bra-side HRR by
 * recursion (a,b+1_i| = (a+1_i,b| + AB_i (a,b|, AB = A - B. */
typedef struct {
    const double* G;
    int nf;
    double AB[3], CD[3];
} HrrCtx;

static double hrr_bra(const HrrCtx* h, int ax, int ay, int az, int bx, int by, int bz, int jf)
{
    if (bx + by + bz == 0) return h->G[(size_t)cidx(ax, ay, az) * h->nf + jf];
    if (bx) return hrr_bra(h, ax + 1, ay, az, bx - 1, by, bz, jf) + h->AB[0] * hrr_bra(h, ax, ay, az, bx - 1, by, bz, jf);
    if (by) return hrr_bra(h, ax, ay + 1, az, bx, by - 1, bz, jf) + h->AB[1] * hrr_bra(h, ax, ay, az, bx, by - 1, bz, jf);
    return hrr_bra(h, ax, ay, az + 1, bx, by, bz - 1, jf) + h->AB[2] * hrr_bra(h, ax, ay, az, bx, by, bz - 1, jf);
}
static double hrr_full(const HrrCtx* h, const int* a, const int* b, int cx, int cy, int cz, int dx, int dy, int dz)
{
    if (dx + dy + dz == 0) return hrr_bra(h, a[0], a[1], a[2], b[0], b[1], b[2], cidx(cx, cy, cz));
    if (dx) return hrr_full(h, a, b, cx + 1, cy, cz, dx - 1, dy, dz) + h->CD[0] * hrr_full(h, a, b, cx, cy, cz, dx - 1, dy, dz);
    if (dy) return hrr_full(h, a, b, cx, cy + 1, cz, dx, dy - 1, dz) + h->CD[1] * hrr_full(h, a, b, cx, cy, cz, dx, dy - 1, dz);
    return hrr_full(h, a, b, cx, cy, cz + 1, dx, dy, dz - 1) + h->CD[2] * hrr_full(h, a, b, cx, cy, cz, dx, dy, dz - 1);
}

/* ---------------------------------------------- contracted shell quartet */
#define X0SQ_GPU 34.986836655249725 /* 2 pi^2.5: product of two X0 = sqrt(2 pi^2.5), gpu_common.h:196 */

/* Contracted (ab|cd) over the basis functions of sub-shells
 * (ii,I) (jj,J) (kk,K) (ll,L), times cons() of each function, into
 * out[((i*nJ + j)*nK + k)*nL + l].  Primitive quartets are screened as in
 * iclass (gpu_get2e_subs.h:603-620): kept iff
 * (DNMax*cutPrim(i,j)) * cutPrim(k,l) > primLimit.  With DNMax < 0 no
 * screen is applied.  If only_prim_ij >= 0, bra and ket are restricted to the
 * single primitive pair (only_prim_ij / 16, only_prim_ij % 16) (used for cutPrim).
 * Returns the number of primitive quartets evaluated. */
long oracle_shell_quartet(const OBasis* b, int ii, int jj, int kk, int ll, int I, int J, int K, int L,
                          double DNMax, const double* cutPrim, double primLimit, int only_prim_ij,
                          double* out)
{
    cart_init();
    int Lab = I + J, Lcd = K + L;
    VrrWork w;
    vrr_alloc(&w, Lab, Lcd);
    int ne = ncart_upto(Lab), nf = ncart_upto(Lcd);
    double* G = (double*)calloc((size_t)ne * nf, sizeof(double));
    const double *A = center(b, ii), *B = center(b, jj), *C = center(b, kk), *D = center(b, ll);
    double AB2 = 0, CD2 = 0;
    for (int x = 0; x < 3; x++) { AB2 += (A[x] - B[x]) * (A[x] - B[x]); CD2 += (C[x] - D[x]) * (C[x] - D[x]); }
    long nprimq = 0;
    for (int pj = 0; pj < b->kprim[jj]; pj++)
        for (int pi = 0; pi < b->kprim[ii]; pi++) {
            if (only_prim_ij >= 0 && (pi != only_prim_ij / 16 || pj != only_prim_ij % 16)) continue;
            double ea = cexpo(b, ii, pi), eb = cexpo(b, jj, pj);
            double Kab = exp(-ea * eb / (ea + eb) * AB2) / (ea + eb) * ccoef(b, ii, I, pi) * ccoef(b, jj, J, pj);
            double cpij = (DNMax >= 0) ? DNMax * F2(cutPrim, b->kstart[ii] - 1 + pi, b->kstart[jj] - 1 + pj, b->jbasis) : 0;
            for (int pl = 0; pl < b->kprim[ll]; pl++)
                for (int pk = 0; pk < b->kprim[kk]; pk++) {
                    if (only_prim_ij >= 0 && (pk != pi || pl != pj)) continue;
                    if (DNMax >= 0 && !(cpij * F2(cutPrim, b->kstart[kk] - 1 + pk, b->kstart[ll] - 1 + pl, b->jbasis) > primLimit))
                        continue;
                    double ec = cexpo(b, kk, pk), ed = cexpo(b, ll, pl);
                    double Kcd = exp(-ec * ed / (ec + ed) * CD2) / (ec + ed) * ccoef(b, kk, K, pk) * ccoef(b, ll, L, pl);
                    double pref = X0SQ_GPU * Kab * Kcd / sqrt(ea + eb + ec + ed);
                    vrr_prim(&w, A, C, ea, eb, ec, ed, B, D, pref);
                    nprimq++;
                    for (int ie = I > 0 ? ncart_upto(I - 1) : 0; ie < ne; ie++)
                        for (int jf = K > 0 ? ncart_upto(K - 1) : 0; jf < nf; jf++)
                            G[(size_t)ie * nf + jf] += VA(&w, ie, jf, 0);
                }
        }
    HrrCtx h = {G, nf, {A[0] - B[0], A[1] - B[1], A[2] - B[2]}, {C[0] - D[0], C[1] - D[1], C[2] - D[2]}};
    int a0 = bf_first(b, ii, I), a1 = bf_last(b, ii, I);
    int b0 = bf_first(b, jj, J), b1 = bf_last(b, jj, J);
    int c0 = bf_first(b, kk, K), c1 = bf_last(b, kk, K);
    int d0 = bf_first(b, ll, L), d1 = bf_last(b, ll, L);
    int nJ = b1 - b0 + 1, nK = c1 - c0 + 1, nL = d1 - d0 + 1;
    for (int ia = a0; ia <= a1; ia++)
        for (int ib = b0; ib <= b1; ib++)
            for (int ic = c0; ic <= c1; ic++)
                for (int id = d0; id <= d1; id++) {
                    const int* ka = b->KLMN + 3 * ia;
                    const int* kb = b->KLMN + 3 * ib;
                    const int* kc = b->KLMN + 3 * ic;
                    const int* kd = b->KLMN + 3 * id;
                    double v = hrr_full(&h, ka, kb, kc[0], kc[1], kc[2], kd[0], kd[1], kd[2]);
                    v *= b->cons[ia] * b->cons[ib] * b->cons[ic] * b->cons[id];
                    out[(((size_t)(ia - a0) * nJ + (ib - b0)) * nK + (ic - c0)) * nL + (id - d0)] = v;
                }
    free(G);
    free(w.A);
    return nprimq;
}

/* ---------------------------------------------------------- Schwarz */
/* YCutoff(II,JJ) = sqrt(max |(ij|ij)|) over the sub-shells and components
 * of shells II, JJ (schwarz.f90:12-42, 46-209, 213-383) and
 * cutPrim(i,j) = sqrt(X0 * max |(ij|ij)_prim|) for each primitive pair
 * (classprim, schwarz.f90:385-548; X0 = 2 pi^2.5 enters squared there).
 * cutPrim is set for primitive pairs of shells II <= JJ only, as in QUICK. */
void oracle_schwarz(const OBasis* b, double* YCutoff, double* cutPrim)
{
    cart_init();
    int ns = b->nshell;
    const double X0F = 2.0 * pow(PI_, 2.5);
    memset(YCutoff, 0, sizeof(double) * ns * ns);
    memset(cutPrim, 0, sizeof(double) * b->jbasis * b->jbasis);
#pragma omp parallel for schedule(dynamic)
    for (int II = 0; II < ns; II++) {
        double buf[10 * 10 * 10 * 10];
        for (int JJ = II; JJ < ns; JJ++) {
            double ymax = 0.0;
            for (int I = b->Qstart[II]; I <= b->Qfinal[II]; I++)
                for (int J = b->Qstart[JJ]; J <= b->Qfinal[JJ]; J++) {
                    oracle_shell_quartet(b, II, JJ, II, JJ, I, J, I, J, -1.0, NULL, 0.0, -1, buf);
                    int nI = bf_last(b, II, I) - bf_first(b, II, I) + 1;
                    int nJ = bf_last(b, JJ, J) - bf_first(b, JJ, J) + 1;
                    for (int x = 0; x < nI; x++)
                        for (int y = 0; y < nJ; y++) {
                            double v = fabs(buf[((x * nJ + y) * nI + x) * nJ + y]);
                            if (v > ymax) ymax = v;
                        }
                }
            YCutoff[II + JJ * ns] = YCutoff[JJ + II * ns] = sqrt(ymax);
            for (int pi = 0; pi < b->kprim[II]; pi++)
                for (int pj = 0; pj < b->kprim[JJ]; pj++) {
                    double pmax = 0.0;
                    for (int I = b->Qstart[II]; I <= b->Qfinal[II]; I++)
                        for (int J = b->Qstart[JJ]; J <= b->Qfinal[JJ]; J++) {
                            oracle_shell_quartet(b, II, JJ, II, JJ, I, J, I, J, -1.0, NULL, 0.0, pi * 16 + pj, buf);
                            int nI = bf_last(b, II, I) - bf_first(b, II, I) + 1;
                            int nJ = bf_last(b, JJ, J) - bf_first(b, JJ, J) + 1;
                            for (int x = 0; x < nI; x++)
                                for (int y = 0; y < nJ; y++) {
                                    double v = fabs(buf[((x * nJ + y) * nI + x) * nJ + y]);
                                    if (v > pmax) pmax = v;
                                }
                        }
                    cutPrim[(b->kstart[II] - 1 + pi) + (size_t)(b->kstart[JJ] - 1 + pj) * b->jbasis] = sqrt(pmax * X0F);
                }
        }
    }
}

/* cutMatrix(II,JJ) = max |D(j,i)| over the functions of shells II, JJ
 * (DNscreen / densityCutoff, schwarz.f90:550-599). */
void oracle_cutmatrix(const OBasis* b, const double* dense, double* cutMatrix)
{
    int ns = b->nshell, nb = b->nbasis;
    for (int II = 0; II < ns; II++)
        for (int JJ = II; JJ < ns; JJ++) {
            int i0 = bf_first(b, II, b->Qstart[II]), i1 = bf_last(b, II, b->Qfinal[II]);
            int j0 = bf_first(b, JJ, b->Qstart[JJ]), j1 = bf_last(b, JJ, b->Qfinal[JJ]);
            double m = 0.0;
            for (int i = i0; i <= i1; i++)
                for (int j = j0; j <= j1; j++) {
                    double v = fabs(dense[j + (size_t)i * nb]);
                    if (v > m) m = v;
                }
            cutMatrix[II + JJ * ns] = cutMatrix[JJ + II * ns] = m;
        }
}

/* ------------------------------------------------------------ Fock */
/* addint's six scatters (gpu_get2e_subs.h:1296-1384) in double precision.
 * III..LLL are 1-based; o is the lower triangle o(row>=col), column-major. */
static void addint_d(double* o, double Y, int III, int JJJ, int KKK, int LLL, double h, const double* D, int n)
{
#define DN(a, b) D[((a) - 1) + (size_t)((b) - 1) * n]
#define OO(a, b) o[((a) - 1) + (size_t)((b) - 1) * n]
    double DKI = DN(KKK, III), DKJ = DN(KKK, JJJ), DLJ = DN(LLL, JJJ), DLI = DN(LLL, III), DLK = DN(LLL, KKK), DJI = DN(JJJ, III);
    OO(JJJ, III) += (KKK == LLL ? 1.0 : 2.0) * DLK * Y;
    if (LLL != JJJ || III != KKK) OO(LLL, KKK) += (III == JJJ ? 1.0 : 2.0) * DJI * Y;
    double v3 = h * 0.5 * DLJ * Y;
    if (III == KKK && III < JJJ && JJJ < LLL) v3 *= 2.0;
    OO(KKK, III) -= v3;
    if (KKK != LLL) OO(LLL, III) -= h * 0.5 * DKJ * Y;
    double v5 = h * 0.5 * DLI * Y;
    if ((III != JJJ && III < KKK) || (III == JJJ && III == KKK && III < LLL) || (III == KKK && III < JJJ && JJJ < LLL)) {
        int r = JJJ > KKK ? JJJ : KKK, c = JJJ > KKK ? KKK : JJJ;
        OO(r, c) -= v5;
    }
    if (III != JJJ && JJJ == KKK) OO(JJJ, KKK) -= v5;
    if (III != JJJ && KKK != LLL) {
        double v6 = h * 0.5 * DKI * Y;
        int r = JJJ > LLL ? JJJ : LLL, c = JJJ > LLL ? LLL : JJJ;
        OO(r, c) -= v6;
        if (JJJ == LLL && III != KKK) OO(LLL, JJJ) -= v6;
    }
#undef DN
#undef OO
}

/* Qshell-level description of the pair set: sorted_Q / sorted_Qnumber
 * (shell index, angular momentum) per Qshell, and the list of kept pairs
 * (x, y) over Qshells.  Only membership matters to the Fock matrix; the
 * order of pairs is checked separately against QUICK's own bridge. */
typedef struct {
    int nq;
    int *qshell, *qL;
    int npair;
    int *px, *py;
} OPairs;

static void build_pairs(const OBasis* b, const double* YCutoff, OPairs* P)
{
    int ns = b->nshell;
    P->nq = 0;
    for (int s = 0; s < ns; s++) P->nq += b->Qfinal[s] - b->Qstart[s] + 1;
    P->qshell = (int*)malloc(sizeof(int) * P->nq);
    P->qL = (int*)malloc(sizeof(int) * P->nq);
    /* stable order by angular momentum (gpu.cu:1191-1218) */
    int q = 0;
    for (int L = 0; L <= MAXL; L++)
        for (int s = 0; s < ns; s++)
            if (b->Qstart[s] <= L && L <= b->Qfinal[s]) { P->qshell[q] = s; P->qL[q] = L; q++; }
    P->px = (int*)malloc(sizeof(int) * (size_t)P->nq * P->nq);
    P->py = (int*)malloc(sizeof(int) * (size_t)P->nq * P->nq);
    P->npair = 0;
    for (int x = 0; x < P->nq; x++)
        for (int y = 0; y < P->nq; y++) {
            int i = P->qshell[x], j = P->qshell[y];
            if (i <= j && YCutoff[i + j * ns] > 1e-10) { P->px[P->npair] = x; P->py[P->npair] = y; P->npair++; }
        }
}

/* Two-electron Fock build.  O (nbasis x nbasis, column-major) is updated in
 * place to O + G(D), symmetric, as gpu_get2e_ returns it (gpu.cu:1806-1864).
 * hybrid: exchange fraction (1 HF, 0.2 B3LYP, 0 pure DFT).  Returns the
 * number of shell quartets (iclass calls); *nprimq gets primitive quartets,
 * *nint the number of integrals passed to addint. */
long oracle_fock(const OBasis* b, const double* YCutoff, const double* cutPrim, const double* cutMatrix,
                 const double* dense, double integralCutoff, double primLimit, double hybrid, double* O,
                 long* nprimq_out, long* nint_out)
{
    cart_init();
    int ns = b->nshell, nb = b->nbasis;
    OPairs P;
    build_pairs(b, YCutoff, &P);
    long nquart = 0, nprimq = 0, nint = 0;
    double* lower = (double*)calloc((size_t)nb * nb, sizeof(double));
#pragma omp parallel reduction(+ : nquart, nprimq, nint)
    {
        double* mine = (double*)calloc((size_t)nb * nb, sizeof(double));
        double* buf = (double*)malloc(sizeof(double) * 10 * 10 * 10 * 10);
#pragma omp for schedule(dynamic, 4)
        for (int a = 0; a < P.npair; a++)
            for (int bb = 0; bb < P.npair; bb++) {
                int II = P.px[a], JJ = P.py[a], KK = P.px[bb], LL = P.py[bb];
                int ii = P.qshell[II], jj = P.qshell[JJ], kk = P.qshell[KK], ll = P.qshell[LL];
                if (ii > kk) continue;
#define CM(x, y) cutMatrix[(x) + (size_t)(y) * ns]
#define MX(x, y) ((x) >= (y) ? (x) : (y))
                double DNMax = MX(MX(4.0 * CM(ii, jj), 4.0 * CM(kk, ll)), MX(MX(CM(ii, ll), CM(ii, kk)), MX(CM(jj, kk), CM(jj, ll))));
                double yy = YCutoff[kk + (size_t)ll * ns] * YCutoff[ii + (size_t)jj * ns];
                if (!(yy > integralCutoff && yy * DNMax > integralCutoff)) continue;
                nquart++;
                int I = P.qL[II], J = P.qL[JJ], K = P.qL[KK], L = P.qL[LL];
                nprimq += oracle_shell_quartet(b, ii, jj, kk, ll, I, J, K, L, DNMax, cutPrim, primLimit, -1, buf);
                int a0 = bf_first(b, ii, I) + 1, a1 = bf_last(b, ii, I) + 1;
                int b0 = bf_first(b, jj, J) + 1, b1 = bf_last(b, jj, J) + 1;
                int c0 = bf_first(b, kk, K) + 1, c1 = bf_last(b, kk, K) + 1;
                int d0 = bf_first(b, ll, L) + 1, d1 = bf_last(b, ll, L) + 1;
                int nJ = b1 - b0 + 1, nK = c1 - c0 + 1, nL = d1 - d0 + 1;
                for (int III = a0; III <= a1; III++)
                    for (int JJJ = MX(III, b0); JJJ <= b1; JJJ++)
                        for (int KKK = MX(III, c0); KKK <= c1; KKK++)
                            for (int LLL = MX(KKK, d0); LLL <= d1; LLL++) {
                                if (III < KKK || (III == JJJ && III == LLL) || (III == JJJ && III < LLL) ||
                                    (JJJ == LLL && III < JJJ) || (III == KKK && III < JJJ && JJJ < LLL)) {
                                    double Y = buf[(((size_t)(III - a0) * nJ + (JJJ - b0)) * nK + (KKK - c0)) * nL + (LLL - d0)];
                                    if (fabs(Y) > 0.0) {
                                        addint_d(mine, Y, III, JJJ, KKK, LLL, hybrid, dense, nb);
                                        nint++;
                                    }
                                }
                            }
            }
#pragma omp critical
        for (size_t k = 0; k < (size_t)nb * nb; k++) lower[k] += mine[k];
        free(mine);
        free(buf);
    }
    for (int i = 0; i < nb; i++)
        for (int j = i; j < nb; j++) {
            double v = lower[j + (size_t)i * nb];
            O[i + (size_t)j * nb] += v;
            if (i != j) O[j + (size_t)i * nb] += v;
        }
    free(lower);
    free(P.qshell); free(P.qL); free(P.px); free(P.py);
    if (nprimq_out) *nprimq_out = nprimq;
    if (nint_out) *nint_out = nint;
    return nquart;
}

/* ------------------------------------------------ derivative integrals */
/* d/dA, d/dB, d/dC of the contracted block (ab|cd) (cons included), laid out
 * as out[3 * (((i*nJ + j)*nK + k)*nL + l) + x].  See oracle_grad.c. */
long oracle_shell_quartet_deriv(const OBasis* b, int ii, int jj, int kk, int ll, int I, int J, int K, int L,
                                double DNMax, const double* cutPrim, double primLimit, double* dA, double* dB,
                                double* dC)
{
    cart_init();
    int Lab = I + J + 1, Lcd = K + L + 1;
    VrrWork w;
    vrr_alloc(&w, Lab, Lcd);
    int ne = ncart_upto(Lab), nf = ncart_upto(Lcd);
    size_t nG = (size_t)ne * nf;
    double* G0 = (double*)calloc(4 * nG, sizeof(double));
    double *GA = G0 + nG, *GB = G0 + 2 * nG, *GC = G0 + 3 * nG;
    const double *A = center(b, ii), *B = center(b, jj), *C = center(b, kk), *D = center(b, ll);
    double AB2 = 0, CD2 = 0;
    for (int x = 0; x < 3; x++) { AB2 += (A[x] - B[x]) * (A[x] - B[x]); CD2 += (C[x] - D[x]) * (C[x] - D[x]); }
    long nprimq = 0;
    for (int pj = 0; pj < b->kprim[jj]; pj++)
        for (int pi = 0; pi < b->kprim[ii]; pi++) {
            double ea = cexpo(b, ii, pi), eb = cexpo(b, jj, pj);
            double Kab = exp(-ea * eb / (ea + eb) * AB2) / (ea + eb) * ccoef(b, ii, I, pi) * ccoef(b, jj, J, pj);
            double cpij = DNMax * F2(cutPrim, b->kstart[ii] - 1 + pi, b->kstart[jj] - 1 + pj, b->jbasis);
            for (int pl = 0; pl < b->kprim[ll]; pl++)
                for (int pk = 0; pk < b->kprim[kk]; pk++) {
                    if (!(cpij * F2(cutPrim, b->kstart[kk] - 1 + pk, b->kstart[ll] - 1 + pl, b->jbasis) > primLimit)) continue;
                    double ec = cexpo(b, kk, pk), ed = cexpo(b, ll, pl);
                    double Kcd = exp(-ec * ed / (ec + ed) * CD2) / (ec + ed) * ccoef(b, kk, K, pk) * ccoef(b, ll, L, pl);
                    double pref = X0SQ_GPU * Kab * Kcd / sqrt(ea + eb + ec + ed);
                    vrr_prim(&w, A, C, ea, eb, ec, ed, B, D, pref);
                    nprimq++;
                    for (size_t ie = 0; ie < (size_t)ne; ie++)
                        for (size_t jf = 0; jf < (size_t)nf; jf++) {
                            double v = VA(&w, ie, jf, 0);
                            G0[ie * nf + jf] += v;
                            GA[ie * nf + jf] += 2.0 * ea * v;
                            GB[ie * nf + jf] += 2.0 * eb * v;
                            GC[ie * nf + jf] += 2.0 * ec * v;
                        }
                }
        }
    HrrCtx h0 = {G0, nf, {A[0] - B[0], A[1] - B[1], A[2] - B[2]}, {C[0] - D[0], C[1] - D[1], C[2] - D[2]}};
    HrrCtx hA = h0, hB = h0, hC = h0;
    hA.G = GA; hB.G = GB; hC.G = GC;
    int a0 = bf_first(b, ii, I), a1 = bf_last(b, ii, I);
    int b0 = bf_first(b, jj, J), b1 = bf_last(b, jj, J);
    int c0 = bf_first(b, kk, K), c1 = bf_last(b, kk, K);
    int d0 = bf_first(b, ll, L), d1 = bf_last(b, ll, L);
    int nJ = b1 - b0 + 1, nK = c1 - c0 + 1, nL = d1 - d0 + 1;
    for (int ia = a0; ia <= a1; ia++)
        for (int ib = b0; ib <= b1; ib++)
            for (int ic = c0; ic <= c1; ic++)
                for (int id = d0; id <= d1; id++) {
                    const int* ka = b->KLMN + 3 * ia;
                    const int* kb = b->KLMN + 3 * ib;
                    const int* kc = b->KLMN + 3 * ic;
                    const int* kd = b->KLMN + 3 * id;
                    double cf = b->cons[ia] * b->cons[ib] * b->cons[ic] * b->cons[id];
                    size_t o = 3 * ((((size_t)(ia - a0) * nJ + (ib - b0)) * nK + (ic - c0)) * nL + (id - d0));
                    for (int x = 0; x < 3; x++) {
                        int ap[3] = {ka[0], ka[1], ka[2]}, am[3] = {ka[0], ka[1], ka[2]};
                        int bp[3] = {kb[0], kb[1], kb[2]}, bm[3] = {kb[0], kb[1], kb[2]};
                        int cp[3] = {kc[0], kc[1], kc[2]}, cmm[3] = {kc[0], kc[1], kc[2]};
                        ap[x]++; am[x]--; bp[x]++; bm[x]--; cp[x]++; cmm[x]--;
                        double va = hrr_full(&hA, ap, kb, kc[0], kc[1], kc[2], kd[0], kd[1], kd[2]);
                        if (ka[x] > 0) va -= ka[x] * hrr_full(&h0, am, kb, kc[0], kc[1], kc[2], kd[0], kd[1], kd[2]);
                        double vb = hrr_full(&hB, ka, bp, kc[0], kc[1], kc[2], kd[0], kd[1], kd[2]);
                        if (kb[x] > 0) vb -= kb[x] * hrr_full(&h0, ka, bm, kc[0], kc[1], kc[2], kd[0], kd[1], kd[2]);
                        double vc = hrr_full(&hC, ka, kb, cp[0], cp[1], cp[2], kd[0], kd[1], kd[2]);
                        if (kc[x] > 0) vc -= kc[x] * hrr_full(&h0, ka, kb, cmm[0], cmm[1], cmm[2], kd[0], kd[1], kd[2]);
                        dA[o + x] = cf * va;
                        dB[o + x] = cf * vb;
                        dC[o + x] = cf * vc;
                    }
                }
    free(G0);
    free(w.A);
    return nprimq;
}
