/*
 * One-electron integrals for the SCF glue around the J/K engine: overlap,
 * kinetic energy and nuclear attraction over Cartesian Gaussians in libcint
 * normalisation (s/p common factors applied, coefficients from env), by the
 * Obara-Saika recursions.  Host code (OpenMP); the SCF driver calls them once
 * per geometry.  PySCF provides these for the reference (mol.intor), outside
 * the reference repository.
 *
 * Output: (nao_cart, nao_cart) row-major over all contractions of all shells,
 * in ao_loc(cart) order.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ATM_SLOTS 6
#define CHARGE_OF 0
#define PTR_COORD 1
#define BAS_SLOTS 8
#define ATOM_OF 0
#define ANG_OF 1
#define NPRIM_OF 2
#define NCTR_OF 3
#define PTR_EXP 5
#define PTR_COEFF 6
#define LM 8 /* max l + 2 (kinetic needs l+1) */

static double fac_sp(int l) { return l == 0 ? 0.282094791773878143 : (l == 1 ? 0.488602511902919921 : 1.0); }

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

static void cart(int l, int c, int *x, int *y, int *z) {
    int n = 0;
    for (int a = l; a >= 0; a--)
        for (int b = l - a; b >= 0; b--) {
            if (n == c) { *x = a; *y = b; *z = l - a - b; return; }
            n++;
        }
}

/* 1D overlap table s[i][j], i <= li+1, j <= lj+1 (unnormalised, without
 * the exp prefactor and (pi/p)^1/2) */
static void ovlp_1d(double pa, double pb, double p, int li, int lj, double s[LM][LM]) {
    memset(s, 0, sizeof(double) * LM * LM);
    s[0][0] = 1;
    double h = 0.5 / p;
    for (int i = 0; i <= li; i++)
        for (int j = 0; j <= lj; j++) {
            if (i == 0 && j == 0) continue;
            if (i > 0) {
                double v = pa * s[i - 1][j];
                if (i > 1) v += (i - 1) * h * s[i - 2][j];
                if (j > 0) v += j * h * s[i - 1][j - 1];
                s[i][j] = v;
            } else {
                double v = pb * s[i][j - 1];
                if (j > 1) v += (j - 1) * h * s[i][j - 2];
                s[i][j] = v;
            }
        }
}

/* Boys function F_m(x), m = 0..mmax: series for the top order, downward
 * recursion; for large x the upward recursion from the asymptotic F_0. */
static void boys(int mmax, double x, double *f) {
    if (x < 35.0) {
        double term = 1.0 / (2 * mmax + 1), sum = term;
        for (int i = 1; i < 500; i++) {
            term *= 2 * x / (2 * mmax + 2 * i + 1);
            sum += term;
            if (term < 1e-17 * sum) break;
        }
        double ex = exp(-x);
        f[mmax] = ex * sum;
        for (int m = mmax - 1; m >= 0; m--) f[m] = (2 * x * f[m + 1] + ex) / (2 * m + 1);
    } else {
        double ex = exp(-x);
        f[0] = 0.5 * sqrt(M_PI / x) * erf(sqrt(x));
        for (int m = 0; m < mmax; m++) f[m + 1] = ((2 * m + 1) * f[m] - ex) / (2 * x);
    }
}

/* nuclear attraction of one primitive pair: out[ci][cj] += sum_C -Z_C <i|1/r_C|j>
 * via the Obara-Saika recursion on (a|A(m)|b) with auxiliary index m */
static void nuc_prim(int li, int lj, double a, double b, const double *A, const double *B, const int *atm,
                     int natm, const double *env, double scale, double *out, int nfj) {
    double p = a + b, P[3];
    for (int d = 0; d < 3; d++) P[d] = (a * A[d] + b * B[d]) / p;
    double ab2 = 0;
    for (int d = 0; d < 3; d++) ab2 += (A[d] - B[d]) * (A[d] - B[d]);
    double pre = 2 * M_PI / p * exp(-a * b / p * ab2) * scale;
    int L = li + lj;
    /* V[m][ax][ay][az][bx][by][bz] is large; build over index tuples with
     * a straightforward recursion in a scratch array indexed by
     * (ia = cart index of total l_a <= L) only on the bra, then HRR. */
    /* VRR on the bra up to L, then horizontal transfer to j */
    int nc = 0, cidx[13][13][13];
    for (int l = 0; l <= L; l++)
        for (int x = l; x >= 0; x--)
            for (int y = l - x; y >= 0; y--) cidx[x][y][l - x - y] = nc++;
    double *V = malloc(sizeof(double) * nc * (L + 1));
    double *acc = calloc(nc, sizeof(double));
    for (int ia = 0; ia < natm; ia++) {
        const double *Cc = env + atm[ia * ATM_SLOTS + PTR_COORD];
        double Z = atm[ia * ATM_SLOTS + CHARGE_OF];
        double pc2 = 0;
        for (int d = 0; d < 3; d++) pc2 += (P[d] - Cc[d]) * (P[d] - Cc[d]);
        double F[32];
        boys(L, p * pc2, F);
        for (int m = 0; m <= L; m++) V[0 * (L + 1) + m] = F[m];
        for (int l = 1; l <= L; l++)
            for (int x = l; x >= 0; x--)
                for (int y = l - x; y >= 0; y--) {
                    int z = l - x - y, e[3] = {x, y, z}, d = x > 0 ? 0 : (y > 0 ? 1 : 2);
                    int em[3] = {x, y, z};
                    em[d]--;
                    int i1 = cidx[em[0]][em[1]][em[2]];
                    int i2 = -1;
                    if (em[d] > 0) {
                        int e2[3] = {em[0], em[1], em[2]};
                        e2[d]--;
                        i2 = cidx[e2[0]][e2[1]][e2[2]];
                    }
                    int io = cidx[x][y][z];
                    for (int m = 0; m <= L - l; m++) {
                        double v = (P[d] - A[d]) * V[i1 * (L + 1) + m] - (P[d] - Cc[d]) * V[i1 * (L + 1) + m + 1];
                        if (i2 >= 0)
                            v += em[d] / (2 * p) * (V[i2 * (L + 1) + m] - V[i2 * (L + 1) + m + 1]);
                        V[io * (L + 1) + m] = v;
                    }
                    (void)e;
                }
        for (int c = 0; c < nc; c++) acc[c] += -Z * V[c * (L + 1)];
    }
    /* HRR: (a|b+1_d) = (a+1_d|b) + (A_d - B_d)(a|b), evaluated recursively */
    int nfi = ncart(li);
    for (int ci = 0; ci < nfi; ci++)
        for (int cj = 0; cj < nfj; cj++) {
            int ax, ay, az, bx, by, bz;
            cart(li, ci, &ax, &ay, &az);
            cart(lj, cj, &bx, &by, &bz);
            /* expand (a|b) = sum over binomial transfer */
            double sum = 0;
            for (int tx = 0; tx <= bx; tx++)
                for (int ty = 0; ty <= by; ty++)
                    for (int tz = 0; tz <= bz; tz++) {
                        double c = 1;
                        /* C(bx,tx) (A-B)^(bx-tx) ... */
                        double bin = 1;
                        for (int k = 0; k < tx; k++) bin = bin * (bx - k) / (k + 1);
                        c *= bin * pow(A[0] - B[0], bx - tx);
                        bin = 1;
                        for (int k = 0; k < ty; k++) bin = bin * (by - k) / (k + 1);
                        c *= bin * pow(A[1] - B[1], by - ty);
                        bin = 1;
                        for (int k = 0; k < tz; k++) bin = bin * (bz - k) / (k + 1);
                        c *= bin * pow(A[2] - B[2], bz - tz);
                        sum += c * acc[cidx[ax + tx][ay + ty][az + tz]];
                    }
            out[ci * nfj + cj] += pre * sum;
        }
    free(V);
    free(acc);
}

/* which: 0 overlap, 1 kinetic, 2 nuclear attraction */
int jk_int1e_cart(int which, const int *atm, int natm, const int *bas, int nbas, const double *env, double *out) {
    if (which < 0 || which > 2 || !atm || !bas || !env || !out) return 3;
    int *ao_loc = malloc(sizeof(int) * (nbas + 1));
    ao_loc[0] = 0;
    for (int i = 0; i < nbas; i++) {
        int l = bas[i * BAS_SLOTS + ANG_OF];
        if (l > 6) { free(ao_loc); return 2; }
        ao_loc[i + 1] = ao_loc[i] + ncart(l) * bas[i * BAS_SLOTS + NCTR_OF];
    }
    int nao = ao_loc[nbas];
    memset(out, 0, sizeof(double) * (size_t)nao * nao);
#pragma omp parallel for schedule(dynamic, 1)
    for (int ish = 0; ish < nbas; ish++)
        for (int jsh = 0; jsh <= ish; jsh++) {
            int li = bas[ish * BAS_SLOTS + ANG_OF], lj = bas[jsh * BAS_SLOTS + ANG_OF];
            int npi = bas[ish * BAS_SLOTS + NPRIM_OF], npj = bas[jsh * BAS_SLOTS + NPRIM_OF];
            int nci = bas[ish * BAS_SLOTS + NCTR_OF], ncj = bas[jsh * BAS_SLOTS + NCTR_OF];
            const double *ai = env + bas[ish * BAS_SLOTS + PTR_EXP], *aj = env + bas[jsh * BAS_SLOTS + PTR_EXP];
            const double *ci = env + bas[ish * BAS_SLOTS + PTR_COEFF], *cj = env + bas[jsh * BAS_SLOTS + PTR_COEFF];
            const double *A = env + atm[bas[ish * BAS_SLOTS + ATOM_OF] * ATM_SLOTS + PTR_COORD];
            const double *B = env + atm[bas[jsh * BAS_SLOTS + ATOM_OF] * ATM_SLOTS + PTR_COORD];
            int nfi = ncart(li), nfj = ncart(lj);
            double *prim = malloc(sizeof(double) * nfi * nfj);
            double *blk = calloc((size_t)nfi * nfj * nci * ncj, sizeof(double));
            double ab2 = 0;
            for (int d = 0; d < 3; d++) ab2 += (A[d] - B[d]) * (A[d] - B[d]);
            for (int ip = 0; ip < npi; ip++)
                for (int jp = 0; jp < npj; jp++) {
                    double a = ai[ip], b = aj[jp], p = a + b;
                    memset(prim, 0, sizeof(double) * nfi * nfj);
                    if (which == 2) {
                        nuc_prim(li, lj, a, b, A, B, atm, natm, env, 1.0, prim, nfj);
                    } else {
                        double s[3][LM][LM];
                        for (int d = 0; d < 3; d++) {
                            double Pd = (a * A[d] + b * B[d]) / p;
                            ovlp_1d(Pd - A[d], Pd - B[d], p, li + 1, lj + 1, s[d]);
                        }
                        double pre = exp(-a * b / p * ab2) * pow(M_PI / p, 1.5);
                        for (int u = 0; u < nfi; u++)
                            for (int v = 0; v < nfj; v++) {
                                int e[3], f[3];
                                cart(li, u, &e[0], &e[1], &e[2]);
                                cart(lj, v, &f[0], &f[1], &f[2]);
                                double val;
                                if (which == 0) {
                                    val = s[0][e[0]][f[0]] * s[1][e[1]][f[1]] * s[2][e[2]][f[2]];
                                } else {
                                    val = 0;
                                    for (int d = 0; d < 3; d++) {
                                        int i = e[d], j = f[d];
                                        double t = 4 * a * b * s[d][i + 1][j + 1];
                                        if (i > 0 && j > 0) t += i * j * s[d][i - 1][j - 1];
                                        if (j > 0) t -= 2 * a * j * s[d][i + 1][j - 1];
                                        if (i > 0) t -= 2 * b * i * s[d][i - 1][j + 1];
                                        double o = 1;
                                        for (int d2 = 0; d2 < 3; d2++)
                                            if (d2 != d) o *= s[d2][e[d2]][f[d2]];
                                        val += 0.5 * t * o;
                                    }
                                }
                                prim[u * nfj + v] = pre * val;
                            }
                    }
                    for (int kc = 0; kc < nci; kc++)
                        for (int lc = 0; lc < ncj; lc++) {
                            double cc = ci[kc * npi + ip] * cj[lc * npj + jp] * fac_sp(li) * fac_sp(lj);
                            for (int u = 0; u < nfi; u++)
                                for (int v = 0; v < nfj; v++)
                                    blk[((kc * nfi + u) * ncj + lc) * nfj + v] += cc * prim[u * nfj + v];
                        }
                }
            for (int kc = 0; kc < nci; kc++)
                for (int u = 0; u < nfi; u++)
                    for (int lc = 0; lc < ncj; lc++)
                        for (int v = 0; v < nfj; v++) {
                            int r = ao_loc[ish] + kc * nfi + u, c = ao_loc[jsh] + lc * nfj + v;
                            double val = blk[((kc * nfi + u) * ncj + lc) * nfj + v];
                            out[(size_t)r * nao + c] = val;
                            out[(size_t)c * nao + r] = val;
                        }
            free(prim);
            free(blk);
        }
    free(ao_loc);
    return 0;
}
