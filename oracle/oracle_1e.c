/*
 * CPU oracle for QUICK's one-electron integrals, their nuclear gradient and
 * the nuclear repulsion: the host-side pieces a direct SCF needs around the
 * two-electron path, restated so that total energies and full gradients can
 * be checked against QUICK's published HF energies and against finite
 * differences.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU legs may load this file's library, and only as the checker.
 *
 *   - overlap: QUICK's closed form (binomial expansion about P and the
 *     half-integer Gamma products), quick_one_electron_integral.f90:177-301;
 *   - kinetic energy as a sum of overlaps with shifted powers,
 *     quick_one_electron_integral.f90:128-172;
 *   - S and the kinetic part of H over basis functions with dcoeff/aexp,
 *     fullx (:31-46) and get1eO (:1633-1673);
 *   - nuclear attraction by the recursive Obara-Saika scheme of attrecurse
 *     (:1990 onward), driven per shell pair like attrashell (:1816-1925) and
 *     nuclearattra (nuclear.f90:198-221, gccoeff x cons per component);
 *   - nuclear repulsion, getEnergy.f90:36-52;
 *   - the one-electron gradient of hfgrad (gradient.f90:49-249): nuclear
 *     repulsion, -2 W dS and 2 D dT over basis-function pairs on different
 *     atoms, and the attraction derivatives of attrashellopt
 *     (shell.f90:1747-1830) with the operator-centre term taken from
 *     translational invariance, dV/dC = -(dV/dA + dV/dB).
 * The Boys function is oracle_boys (oracle.c), accurate to full precision.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

void oracle_boys(int mmax, double T, double* F);

static const double PI1 = 3.1415926535897932384626433832795;

typedef struct {
    int natom, nbasis, nshell, maxcontract;
    const double* xyz;                  /* (3, natom) bohr */
    const double* chg;                  /* nuclear charges */
    const int *ncontract, *itype, *ncenter;     /* per basis function; itype (3, nbasis); ncenter 1-based */
    const double *aexp, *dcoeff;                /* (maxcontract, nbasis) */
    const int *katom, *kprim, *Ksumtype, *Qstart, *Qfinal, *Qsbasis, *Qfbasis, *KLMN;
    const double *gccoeff, *gcexpo, *cons;      /* gccoeff/gcexpo (10, nbasis) */
} O1Basis;

#define MAXPRIM1 10
#define G2(A, i, j, d1) (A)[(i) + (size_t)(j) * (d1)]

static double fact(int n)
{
    double f = 1.0;
    for (int i = 2; i <= n; i++) f *= i;
    return f;
}

/* quick_one_electron_integral.f90:177-301.  Overlap of the primitive
 * x^i y^j z^k e^{-a r_A^2} with x^ii y^jj z^kk e^{-b r_B^2}. */
double oracle_overlap(double a, double b, int i, int j, int k, int ii, int jj, int kk, const double* A, const double* B)
{
    if (i < 0 || j < 0 || k < 0 || ii < 0 || jj < 0 || kk < 0) return 0.0;
    const double R2 = (A[0] - B[0]) * (A[0] - B[0]) + (A[1] - B[1]) * (A[1] - B[1]) + (A[2] - B[2]) * (A[2] - B[2]);
    const int odd = ((i + ii) & 1) || ((j + jj) & 1) || ((k + kk) & 1);
    if (odd && R2 == 0.0) return 0.0;
    const double g = a + b;
    double P[3], PA[3], PB[3];
    for (int d = 0; d < 3; d++) {
        P[d] = (a * A[d] + b * B[d]) / g;
        PA[d] = P[d] - A[d];
        PB[d] = P[d] - B[d];
    }
    const double xnumfact = fact(i) * fact(ii) * fact(j) * fact(jj) * fact(k) * fact(kk);
    double s = 0.0;
    for (int il = 0; il <= i; il++)
        for (int iil = 0; iil <= ii; iil++)
            for (int jl = 0; jl <= j; jl++)
                for (int jjl = 0; jjl <= jj; jjl++)
                    for (int kl = 0; kl <= k; kl++)
                        for (int kkl = 0; kkl <= kk; kkl++) {
                            const int ix = il + iil, jy = jl + jjl, kz = kl + kkl;
                            if ((ix & 1) || (jy & 1) || (kz & 1)) continue;
                            double e = pow(PA[0], i - il) * pow(PB[0], ii - iil) * pow(PA[1], j - jl) *
                                       pow(PB[1], jj - jjl) * pow(PA[2], k - kl) * pow(PB[2], kk - kkl) * xnumfact /
                                       (fact(il) * fact(iil) * fact(jl) * fact(jjl) * fact(kl) * fact(kkl) *
                                        fact(i - il) * fact(ii - iil) * fact(j - jl) * fact(jj - jjl) *
                                        fact(k - kl) * fact(kk - kkl));
                            e *= pow(g, (double)(-3 - ix - jy - kz) / 2.0);
                            for (int t = 1; t <= ix / 2; t++) e *= ix / 2.0 - t + 0.5;
                            for (int t = 1; t <= jy / 2; t++) e *= jy / 2.0 - t + 0.5;
                            for (int t = 1; t <= kz / 2; t++) e *= kz / 2.0 - t + 0.5;
                            s += e * PI1 * sqrt(PI1);
                        }
    return s * exp(-(a * b * R2) / g);
}

/* quick_one_electron_integral.f90:128-172: -1/2 <(i,j,k) a | nabla^2 ... > as
 * a sum of overlaps with the powers of the first function shifted by -2, 0, +2. */
double oracle_kinetic(double a, double b, int i, int j, int k, int ii, int jj, int kk, const double* A, const double* B)
{
    int e[3] = {i, j, k};
    double t = 0.0;
    for (int d = 0; d < 3; d++) {
        int m[3] = {e[0], e[1], e[2]};
        const double x = e[d];
        m[d] = e[d] - 2;
        t += (x - 1.0) * x * oracle_overlap(a, b, m[0], m[1], m[2], ii, jj, kk, A, B);
        m[d] = e[d];
        t -= 2.0 * a * (1.0 + 2.0 * x) * oracle_overlap(a, b, m[0], m[1], m[2], ii, jj, kk, A, B);
        m[d] = e[d] + 2;
        t += 4.0 * a * a * oracle_overlap(a, b, m[0], m[1], m[2], ii, jj, kk, A, B);
    }
    return t / -2.0;
}

/* Recursive Obara-Saika nuclear attraction (a|1/r_C|b)^(m) from the
 * auxiliary integrals aux[m] = (2 pi / g) K_AB F_m(g PC^2), following
 * attrecurse: lower the first nonzero power of a, else of b. */
typedef struct {
    double PA[3], PB[3], PC[3], o2g;
    const double* aux;
} AttrCtx;

static double attr_rec(const AttrCtx* c, int a0, int a1, int a2, int b0, int b1, int b2, int m)
{
    int a[3] = {a0, a1, a2}, b[3] = {b0, b1, b2};
    int d = -1, onb = 0;
    for (int k = 0; k < 3 && d < 0; k++)
        if (a[k] > 0) d = k;
    if (d < 0) {
        for (int k = 0; k < 3 && d < 0; k++)
            if (b[k] > 0) d = k;
        onb = 1;
    }
    if (d < 0) return c->aux[m];
    int* x = onb ? b : a;          /* the side that is lowered */
    int* y = onb ? a : b;
    const double XP = onb ? c->PB[d] : c->PA[d];
    x[d]--;
    double v = XP * attr_rec(c, a[0], a[1], a[2], b[0], b[1], b[2], m) -
               c->PC[d] * attr_rec(c, a[0], a[1], a[2], b[0], b[1], b[2], m + 1);
    if (x[d] > 0) {
        const double n = x[d];
        x[d]--;
        v += n * c->o2g * (attr_rec(c, a[0], a[1], a[2], b[0], b[1], b[2], m) -
                           attr_rec(c, a[0], a[1], a[2], b[0], b[1], b[2], m + 1));
        x[d]++;
    }
    if (y[d] > 0) {
        const double n = y[d];
        y[d]--;
        v += n * c->o2g * (attr_rec(c, a[0], a[1], a[2], b[0], b[1], b[2], m) -
                           attr_rec(c, a[0], a[1], a[2], b[0], b[1], b[2], m + 1));
        y[d]++;
    }
    return v;
}

static const double* atom_xyz(const O1Basis* B, int atom0) { return B->xyz + 3 * atom0; }

/* S (fullx, :31-46) and H = T (get1eO) + V (attrashell/nuclearattra), full
 * symmetric nbasis x nbasis, column-major. */
void oracle_oneint(const O1Basis* B, double* S, double* H)
{
    const int n = B->nbasis;
    for (int I = 0; I < n; I++)
        for (int J = I; J < n; J++) {
            const double* RA = atom_xyz(B, B->ncenter[I] - 1);
            const double* RB = atom_xyz(B, B->ncenter[J] - 1);
            const int* ti = B->itype + 3 * I;
            const int* tj = B->itype + 3 * J;
            double s = 0.0, t = 0.0;
            for (int ic = 0; ic < B->ncontract[I]; ic++)
                for (int jc = 0; jc < B->ncontract[J]; jc++) {
                    const double f = G2(B->dcoeff, jc, J, B->maxcontract) * G2(B->dcoeff, ic, I, B->maxcontract);
                    const double aj = G2(B->aexp, jc, J, B->maxcontract), ai = G2(B->aexp, ic, I, B->maxcontract);
                    s += f * oracle_overlap(aj, ai, tj[0], tj[1], tj[2], ti[0], ti[1], ti[2], RB, RA);
                    t += f * oracle_kinetic(aj, ai, tj[0], tj[1], tj[2], ti[0], ti[1], ti[2], RB, RA);
                }
            S[J + (size_t)I * n] = S[I + (size_t)J * n] = s;
            H[J + (size_t)I * n] = H[I + (size_t)J * n] = t;
        }
    /* attraction, per shell pair IIsh <= JJsh, lower triangle JJJ >= III */
    double* V = (double*)calloc((size_t)n * n, sizeof(double));
    for (int Ish = 0; Ish < B->nshell; Ish++)
        for (int Jsh = Ish; Jsh < B->nshell; Jsh++) {
            const double* RA = atom_xyz(B, B->katom[Ish] - 1);
            const double* RB = atom_xyz(B, B->katom[Jsh] - 1);
            const double R2 = (RA[0] - RB[0]) * (RA[0] - RB[0]) + (RA[1] - RB[1]) * (RA[1] - RB[1]) +
                              (RA[2] - RB[2]) * (RA[2] - RB[2]);
            const int maxm = B->Qfinal[Ish] + B->Qfinal[Jsh];
            for (int ip = 0; ip < B->kprim[Ish]; ip++)
                for (int jp = 0; jp < B->kprim[Jsh]; jp++) {
                    const double a = G2(B->gcexpo, ip, B->Ksumtype[Ish] - 1, MAXPRIM1);
                    const double b = G2(B->gcexpo, jp, B->Ksumtype[Jsh] - 1, MAXPRIM1);
                    const double g = a + b;
                    double P[3];
                    for (int d = 0; d < 3; d++) P[d] = (a * RA[d] + b * RB[d]) / g;
                    const double K = 2.0 * PI1 / g * exp(-a * b * R2 / g);
                    for (int C = 0; C < B->natom; C++) {
                        const double* RC = atom_xyz(B, C);
                        AttrCtx c;
                        double aux[32], PC2 = 0.0;
                        for (int d = 0; d < 3; d++) {
                            c.PA[d] = P[d] - RA[d];
                            c.PB[d] = P[d] - RB[d];
                            c.PC[d] = P[d] - RC[d];
                            PC2 += c.PC[d] * c.PC[d];
                        }
                        c.o2g = 0.5 / g;
                        oracle_boys(maxm, g * PC2, aux);
                        const double Z = -B->chg[C];
                        for (int m = 0; m <= maxm; m++) aux[m] *= K * Z;
                        c.aux = aux;
                        for (int LI = B->Qstart[Ish]; LI <= B->Qfinal[Ish]; LI++)
                            for (int LJ = B->Qstart[Jsh]; LJ <= B->Qfinal[Jsh]; LJ++) {
                                const double X = G2(B->gccoeff, ip, B->Ksumtype[Ish] - 1 + LI, MAXPRIM1) *
                                                 G2(B->gccoeff, jp, B->Ksumtype[Jsh] - 1 + LJ, MAXPRIM1);
                                const int i1 = B->Ksumtype[Ish] - 1 + G2(B->Qsbasis, Ish, LI, B->nshell);
                                const int i2 = B->Ksumtype[Ish] - 1 + G2(B->Qfbasis, Ish, LI, B->nshell);
                                const int j1 = B->Ksumtype[Jsh] - 1 + G2(B->Qsbasis, Jsh, LJ, B->nshell);
                                const int j2 = B->Ksumtype[Jsh] - 1 + G2(B->Qfbasis, Jsh, LJ, B->nshell);
                                for (int III = i1; III <= i2; III++)
                                    for (int JJJ = (III > j1 ? III : j1); JJJ <= j2; JJJ++) {
                                        const int* ka = B->KLMN + 3 * III;
                                        const int* kb = B->KLMN + 3 * JJJ;
                                        V[JJJ + (size_t)III * n] += X * B->cons[III] * B->cons[JJJ] *
                                            attr_rec(&c, ka[0], ka[1], ka[2], kb[0], kb[1], kb[2], 0);
                                    }
                            }
                    }
                }
        }
    for (int I = 0; I < n; I++)
        for (int J = I; J < n; J++) {
            const double v = V[J + (size_t)I * n];
            H[J + (size_t)I * n] += v;
            if (J != I) H[I + (size_t)J * n] += v;
        }
    free(V);
}

/* getEnergy.f90:36-52 */
double oracle_enuc(int natom, const double* xyz, const double* chg)
{
    double e = 0.0;
    for (int i = 0; i < natom; i++)
        for (int j = i + 1; j < natom; j++) {
            double r2 = 0.0;
            for (int d = 0; d < 3; d++) r2 += (xyz[3 * i + d] - xyz[3 * j + d]) * (xyz[3 * i + d] - xyz[3 * j + d]);
            e += chg[i] * chg[j] / sqrt(r2);
        }
    return e;
}

/* One-electron and nuclear-repulsion parts of the RHF gradient (hfgrad,
 * gradient.f90:49-249), added to grad (3, natom).  D is the total density,
 * W = 2 sum_occ e_k C_k C_k^T the energy-weighted density. */
void oracle_grad1e(const O1Basis* B, const double* D, const double* W, double* grad)
{
    const int n = B->nbasis, na = B->natom;
    /* nuclear repulsion (gradient.f90:57-78) */
    for (int i = 0; i < na; i++)
        for (int j = i + 1; j < na; j++) {
            double d[3], r2 = 0.0;
            for (int k = 0; k < 3; k++) {
                d[k] = B->xyz[3 * j + k] - B->xyz[3 * i + k];
                r2 += d[k] * d[k];
            }
            const double f = B->chg[i] * B->chg[j] * pow(r2, -1.5);
            for (int k = 0; k < 3; k++) {
                grad[3 * i + k] += d[k] * f;
                grad[3 * j + k] -= d[k] * f;
            }
        }
    /* overlap and kinetic derivatives over basis-function pairs on different
     * atoms, Jbas after Ibas's atom (gradient.f90:107-233) */
    for (int I = 0; I < n; I++) {
        const int ai = B->ncenter[I] - 1;
        for (int J = 0; J < n; J++) {
            const int aj = B->ncenter[J] - 1;
            if (aj <= ai) continue;
            const double* RA = atom_xyz(B, ai);
            const double* RB = atom_xyz(B, aj);
            const double DJI = D[J + (size_t)I * n], WJI = W[J + (size_t)I * n];
            for (int d = 0; d < 3; d++) {
                double dSI = 0, dSJ = 0, dKI = 0, dKJ = 0;
                for (int ic = 0; ic < B->ncontract[I]; ic++)
                    for (int jc = 0; jc < B->ncontract[J]; jc++) {
                        const double f = G2(B->dcoeff, jc, J, B->maxcontract) * G2(B->dcoeff, ic, I, B->maxcontract);
                        const double aJ = G2(B->aexp, jc, J, B->maxcontract), aI = G2(B->aexp, ic, I, B->maxcontract);
                        int ti[3] = {B->itype[3 * I], B->itype[3 * I + 1], B->itype[3 * I + 2]};
                        int tj[3] = {B->itype[3 * J], B->itype[3 * J + 1], B->itype[3 * J + 2]};
                        /* d/dA of the I function: 2 a x^(i+1) - i x^(i-1) */
                        int up[3] = {ti[0], ti[1], ti[2]}, dn[3] = {ti[0], ti[1], ti[2]};
                        up[d]++;
                        dn[d]--;
                        dSI += f * 2.0 * aI * oracle_overlap(aJ, aI, tj[0], tj[1], tj[2], up[0], up[1], up[2], RB, RA);
                        dKI += f * 2.0 * aI * oracle_kinetic(aJ, aI, tj[0], tj[1], tj[2], up[0], up[1], up[2], RB, RA);
                        if (ti[d] > 0) {
                            dSI -= f * ti[d] * oracle_overlap(aJ, aI, tj[0], tj[1], tj[2], dn[0], dn[1], dn[2], RB, RA);
                            dKI -= f * ti[d] * oracle_kinetic(aJ, aI, tj[0], tj[1], tj[2], dn[0], dn[1], dn[2], RB, RA);
                        }
                        int uj[3] = {tj[0], tj[1], tj[2]}, dj[3] = {tj[0], tj[1], tj[2]};
                        uj[d]++;
                        dj[d]--;
                        dSJ += f * 2.0 * aJ * oracle_overlap(aJ, aI, uj[0], uj[1], uj[2], ti[0], ti[1], ti[2], RB, RA);
                        dKJ += f * 2.0 * aJ * oracle_kinetic(aJ, aI, uj[0], uj[1], uj[2], ti[0], ti[1], ti[2], RB, RA);
                        if (tj[d] > 0) {
                            dSJ -= f * tj[d] * oracle_overlap(aJ, aI, dj[0], dj[1], dj[2], ti[0], ti[1], ti[2], RB, RA);
                            dKJ -= f * tj[d] * oracle_kinetic(aJ, aI, dj[0], dj[1], dj[2], ti[0], ti[1], ti[2], RB, RA);
                        }
                    }
                grad[3 * ai + d] += -dSI * WJI * 2.0 + dKI * DJI * 2.0;
                grad[3 * aj + d] += -dSJ * WJI * 2.0 + dKJ * DJI * 2.0;
            }
        }
    }
    /* attraction derivatives over all ordered shell pairs and components */
    for (int Ish = 0; Ish < B->nshell; Ish++)
        for (int Jsh = 0; Jsh < B->nshell; Jsh++) {
            const int atA = B->katom[Ish] - 1, atB = B->katom[Jsh] - 1;
            const double* RA = atom_xyz(B, atA);
            const double* RB = atom_xyz(B, atB);
            const double R2 = (RA[0] - RB[0]) * (RA[0] - RB[0]) + (RA[1] - RB[1]) * (RA[1] - RB[1]) +
                              (RA[2] - RB[2]) * (RA[2] - RB[2]);
            const int maxm = B->Qfinal[Ish] + B->Qfinal[Jsh] + 1;
            for (int ip = 0; ip < B->kprim[Ish]; ip++)
                for (int jp = 0; jp < B->kprim[Jsh]; jp++) {
                    const double a = G2(B->gcexpo, ip, B->Ksumtype[Ish] - 1, MAXPRIM1);
                    const double b = G2(B->gcexpo, jp, B->Ksumtype[Jsh] - 1, MAXPRIM1);
                    const double g = a + b;
                    double P[3];
                    for (int d = 0; d < 3; d++) P[d] = (a * RA[d] + b * RB[d]) / g;
                    const double K = 2.0 * PI1 / g * exp(-a * b * R2 / g);
                    for (int C = 0; C < na; C++) {
                        if (C == atA && C == atB) continue;
                        const double* RC = atom_xyz(B, C);
                        AttrCtx c;
                        double aux[32], PC2 = 0.0;
                        for (int d = 0; d < 3; d++) {
                            c.PA[d] = P[d] - RA[d];
                            c.PB[d] = P[d] - RB[d];
                            c.PC[d] = P[d] - RC[d];
                            PC2 += c.PC[d] * c.PC[d];
                        }
                        c.o2g = 0.5 / g;
                        oracle_boys(maxm, g * PC2, aux);
                        const double Z = -B->chg[C];
                        for (int m = 0; m <= maxm; m++) aux[m] *= K * Z;
                        c.aux = aux;
                        for (int LI = B->Qstart[Ish]; LI <= B->Qfinal[Ish]; LI++)
                            for (int LJ = B->Qstart[Jsh]; LJ <= B->Qfinal[Jsh]; LJ++) {
                                const double X = G2(B->gccoeff, ip, B->Ksumtype[Ish] - 1 + LI, MAXPRIM1) *
                                                 G2(B->gccoeff, jp, B->Ksumtype[Jsh] - 1 + LJ, MAXPRIM1);
                                const int i1 = B->Ksumtype[Ish] - 1 + G2(B->Qsbasis, Ish, LI, B->nshell);
                                const int i2 = B->Ksumtype[Ish] - 1 + G2(B->Qfbasis, Ish, LI, B->nshell);
                                const int j1 = B->Ksumtype[Jsh] - 1 + G2(B->Qsbasis, Jsh, LJ, B->nshell);
                                const int j2 = B->Ksumtype[Jsh] - 1 + G2(B->Qfbasis, Jsh, LJ, B->nshell);
                                for (int III = i1; III <= i2; III++)
                                    for (int JJJ = j1; JJJ <= j2; JJJ++) {
                                        const double w = X * B->cons[III] * B->cons[JJJ] * D[III + (size_t)JJJ * n];
                                        if (w == 0.0) continue;
                                        const int* ka = B->KLMN + 3 * III;
                                        const int* kb = B->KLMN + 3 * JJJ;
                                        for (int d = 0; d < 3; d++) {
                                            int au[3] = {ka[0], ka[1], ka[2]}, bu[3] = {kb[0], kb[1], kb[2]};
                                            au[d]++;
                                            bu[d]++;
                                            double gA = 2.0 * a * attr_rec(&c, au[0], au[1], au[2], kb[0], kb[1], kb[2], 0);
                                            double gB = 2.0 * b * attr_rec(&c, ka[0], ka[1], ka[2], bu[0], bu[1], bu[2], 0);
                                            if (ka[d] > 0) {
                                                au[d] -= 2;
                                                gA -= ka[d] * attr_rec(&c, au[0], au[1], au[2], kb[0], kb[1], kb[2], 0);
                                            }
                                            if (kb[d] > 0) {
                                                bu[d] -= 2;
                                                gB -= kb[d] * attr_rec(&c, ka[0], ka[1], ka[2], bu[0], bu[1], bu[2], 0);
                                            }
                                            grad[3 * atA + d] += w * gA;
                                            grad[3 * atB + d] += w * gB;
                                            grad[3 * C + d] -= w * (gA + gB);
                                        }
                                    }
                            }
                    }
                }
        }
}
