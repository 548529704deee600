/*
 * Build-time generator of the Rys quadrature tables used by the J/K kernels.
 *
 * For n roots and x = rho |P-Q|^2 the Rys rule has nodes s_i = t_i^2 in (0,1)
 * and weights w_i with  sum_i w_i s_i^k = F_k(x)  (k < 2n), F_k the Boys
 * function.  The reference evaluates u_i = s_i/(1-s_i) and w_i from
 * interval fits (cuobc/lib/gint/rys_roots.cu:1214-2176, tables in
 * rys_xw.cuh); this generator makes its own tables from first principles:
 *
 *   1. F_k(x) in __float128 by the (positive-term) series for the highest
 *      order and downward recursion;
 *   2. recurrence coefficients of the monic orthogonal polynomials in s by
 *      the ordinary Chebyshev algorithm on the moments F_0..F_{2n-1} (the
 *      conditioning loss, ~1e-16 at n = 11, is absorbed by quad precision);
 *   3. nodes by Sturm-sequence bisection of the Jacobi matrix, weights by
 *      the Christoffel numbers 1 / sum_k p_k(s_i)^2 (orthonormal p_k);
 *   4. on [0, X_n): piecewise Chebyshev series of degree NC-1 on uniform
 *      intervals of width h_n, chosen so that the double-precision Clenshaw
 *      evaluation meets the tolerance below at random check points;
 *   5. for x >= X_n: the half-range Gauss-Hermite limit s_i = y_i^2 / x,
 *      w_i = H_i / sqrt(x) (2n-point Gauss-Hermite, positive nodes), with
 *      X_n the smallest point from which that limit is exact to 2e-17.
 *
 * Output: a C header with hex-float literals (exact doubles).
 * Usage: rys_gen <nmax> <out.h>
 */
#include <math.h>
#include <quadmath.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef __float128 qf;
#define NC 14
#define NMAXG 13

static void boys_q(int mmax, qf x, qf *f) {
    qf term = 1.0Q / (2 * mmax + 1), sum = term;
    for (int i = 1; i < 100000; i++) {
        term *= 2 * x / (2 * mmax + 2 * i + 1);
        sum += term;
        if (term < sum * 1e-40Q) break;
    }
    qf ex = expq(-x);
    f[mmax] = ex * sum;
    for (int m = mmax - 1; m >= 0; m--) f[m] = (2 * x * f[m + 1] + ex) / (2 * m + 1);
}

/* eigenvalues of the symmetric tridiagonal matrix (diag a, off-diag sqrt(b[1..]))
 * in [lo, hi] by bisection; returns them ascending. */
static int sturm_count(int n, const qf *a, const qf *b, qf lam) {
    int cnt = 0;
    qf d = a[0] - lam;
    if (d < 0) cnt++;
    for (int k = 1; k < n; k++) {
        if (d == 0) d = 1e-60Q;
        d = a[k] - lam - b[k] / d;
        if (d < 0) cnt++;
    }
    return cnt;
}

static void jacobi_eig(int n, const qf *a, const qf *b, qf lo, qf hi, qf *ev) {
    for (int i = 0; i < n; i++) {
        qf l = lo, h = hi;
        for (int it = 0; it < 400; it++) {
            qf m = (l + h) / 2;
            if (m == l || m == h) break;
            if (sturm_count(n, a, b, m) > i) h = m; else l = m;
        }
        ev[i] = (l + h) / 2;
    }
}

/* Christoffel weights from the recurrence (a = alpha, b = beta, b[0] = mu0) */
static void christoffel(int n, const qf *a, const qf *b, const qf *s, qf *w) {
    for (int i = 0; i < n; i++) {
        qf pm1 = 0, p = 1 / sqrtq(b[0]), sum = p * p;
        for (int k = 0; k < n - 1; k++) {
            qf pn = ((s[i] - a[k]) * p - (k > 0 ? sqrtq(b[k]) * pm1 : 0)) / sqrtq(b[k + 1]);
            pm1 = p;
            p = pn;
            sum += p * p;
        }
        w[i] = 1 / sum;
    }
}

/* exact Rys nodes/weights in quad precision */
static void rys_exact(int n, qf x, qf *s, qf *w) {
    qf mu[2 * NMAXG], a[NMAXG], b[NMAXG];
    qf sig0[2 * NMAXG], sig1[2 * NMAXG], sig2[2 * NMAXG];
    boys_q(2 * n - 1, x, mu);
    a[0] = mu[1] / mu[0];
    b[0] = mu[0];
    for (int l = 0; l < 2 * n; l++) { sig1[l] = mu[l]; sig0[l] = 0; }
    for (int k = 1; k < n; k++) {
        for (int l = k; l < 2 * n - k; l++)
            sig2[l] = sig1[l + 1] - a[k - 1] * sig1[l] - b[k - 1] * sig0[l];
        a[k] = sig2[k + 1] / sig2[k] - sig1[k] / sig1[k - 1];
        b[k] = sig2[k] / sig1[k - 1];
        memcpy(sig0, sig1, sizeof(sig1));
        memcpy(sig1, sig2, sizeof(sig2));
    }
    jacobi_eig(n, a, b, 0, 1, s);
    christoffel(n, a, b, s, w);
}

/* positive nodes y_i^2 and weights H_i of the 2n-point Gauss-Hermite rule */
static void hermite_half(int n, qf *r, qf *hw) {
    int m = 2 * n;
    qf a[2 * NMAXG], b[2 * NMAXG], y[2 * NMAXG], w[2 * NMAXG];
    for (int k = 0; k < m; k++) { a[k] = 0; b[k] = k / 2.0Q; }
    b[0] = sqrtq(M_PIq);
    jacobi_eig(m, a, b, -20, 20, y);
    christoffel(m, a, b, y, w);
    for (int i = 0; i < n; i++) { r[i] = y[n + i] * y[n + i]; hw[i] = w[n + i]; }
}

static void cheb_fit(int n, qf x0, qf h, double *coef /* [2n][NC] */) {
    qf fs[NC][2 * NMAXG];
    for (int j = 0; j < NC; j++) {
        qf t = cosq(M_PIq * (j + 0.5Q) / NC);
        qf x = x0 + h / 2 + h / 2 * t;
        qf s[NMAXG], w[NMAXG];
        rys_exact(n, x, s, w);
        for (int i = 0; i < n; i++) { fs[j][i] = s[i]; fs[j][n + i] = w[i]; }
    }
    for (int f = 0; f < 2 * n; f++)
        for (int k = 0; k < NC; k++) {
            qf acc = 0;
            for (int j = 0; j < NC; j++) acc += fs[j][f] * cosq(M_PIq * k * (j + 0.5Q) / NC);
            acc *= 2.0Q / NC;
            if (k == 0) acc /= 2;
            coef[f * NC + k] = (double)acc;
        }
}

static double clenshaw(const double *c, double t) {
    double b1 = 0, b2 = 0, t2 = 2 * t;
    for (int k = NC - 1; k >= 1; k--) {
        double b0 = fma(t2, b1, c[k] - b2);
        b2 = b1;
        b1 = b0;
    }
    return fma(t, b1, c[0] - b2);
}

static unsigned long long rng_state = 88172645463325252ULL;
static double urand(void) {
    rng_state ^= rng_state << 13;
    rng_state ^= rng_state >> 7;
    rng_state ^= rng_state << 17;
    return (rng_state >> 11) * (1.0 / 9007199254740992.0);
}

/* tolerances for the double evaluation of a fit */
#define TOL_S 4e-15 /* relative, per node */
#define TOL_W 1e-15 /* relative to F_0(x) */

static double fit_error(int n, qf x0, qf h, const double *coef) {
    double worst = 0;
    for (int r = 0; r < 6; r++) {
        double t = 2 * urand() - 1;
        qf x = x0 + h / 2 + h / 2 * (qf)t;
        qf s[NMAXG], w[NMAXG];
        rys_exact(n, x, s, w);
        qf f0 = 0;
        for (int i = 0; i < n; i++) f0 += w[i];
        for (int i = 0; i < n; i++) {
            double es = fabs(clenshaw(coef + i * NC, t) - (double)s[i]) / (double)s[i];
            double ew = fabs(clenshaw(coef + (n + i) * NC, t) - (double)w[i]) / (double)f0;
            if (es / TOL_S > worst) worst = es / TOL_S;
            if (ew / TOL_W > worst) worst = ew / TOL_W;
        }
    }
    return worst;
}

/* smallest X (on a 1.0 grid) from which the Hermite limit holds */
static double asymptote_start(int n, const qf *r, const qf *hw) {
    double x = 8;
    for (;; x += 1) {
        int ok = 1;
        for (double xx = x; xx < x + 40; xx += 2.5) {
            qf s[NMAXG], w[NMAXG];
            rys_exact(n, xx, s, w);
            qf f0 = 0;
            for (int i = 0; i < n; i++) f0 += w[i];
            for (int i = 0; i < n; i++) {
                qf sa = r[i] / xx, wa = hw[i] / sqrtq(xx);
                if (fabsq(sa - s[i]) / s[i] > 2e-17Q || fabsq(wa - w[i]) / f0 > 2e-17Q) ok = 0;
            }
        }
        if (ok) return x;
    }
}

int main(int argc, char **argv) {
    if (argc < 3) { fprintf(stderr, "usage: %s nmax out.h\n", argv[0]); return 2; }
    int nmax = atoi(argv[1]);
    if (nmax < 1 || nmax > NMAXG) return 2;
    FILE *fo = fopen(argv[2], "w");
    if (!fo) return 1;
    double hs[NMAXG + 1];
    int nint[NMAXG + 1], off[NMAXG + 2];
    double *tables[NMAXG + 1];
    double xas[NMAXG + 1];
    qf hr[NMAXG + 1][NMAXG], hh[NMAXG + 1][NMAXG];
    off[1] = 0;
    for (int n = 1; n <= nmax; n++) {
        hermite_half(n, hr[n], hh[n]);
        double xa = asymptote_start(n, hr[n], hh[n]);
        /* widest interval (from a ladder) whose fit passes everywhere */
        static const double ladder[] = {4.0, 2.0, 1.0, 0.5, 0.25};
        for (int il = 0; il < 5; il++) {
            double h = ladder[il];
            int m = (int)ceil(xa / h);
            double *tab = malloc(sizeof(double) * m * 2 * n * NC);
            double worst = 0;
            for (int k = 0; k < m; k++) {
                cheb_fit(n, k * (qf)h, h, tab + (size_t)k * 2 * n * NC);
                double e = fit_error(n, k * (qf)h, h, tab + (size_t)k * 2 * n * NC);
                if (e > worst) worst = e;
            }
            if (worst <= 1.0 || il == 4) {
                hs[n] = h; nint[n] = m; tables[n] = tab; xas[n] = m * h;
                fprintf(stderr, "n=%2d h=%.2f intervals=%3d X=%.1f worst/tol=%.3f\n", n, h, m, m * h, worst);
                break;
            }
            free(tab);
        }
        off[n + 1] = off[n] + nint[n] * 2 * n * NC;
    }
    fprintf(fo, "/* generated by rys_gen.c: Rys nodes s=t^2 and weights, %d-term Chebyshev\n"
                " * series on uniform intervals, Gauss-Hermite limit beyond.  The small\n"
                " * metadata arrays use RYS_META storage; the coefficient array is emitted\n"
                " * only where RYS_WANT_COEF is defined (one host translation unit). */\n", NC);
    fprintf(fo, "#define RYS_NC %d\n#define RYS_NMAX %d\n#define RYS_TOTAL %d\n", NC, nmax, off[nmax + 1]);
    fprintf(fo, "#ifndef RYS_META\n#define RYS_META static const\n#endif\n");
    fprintf(fo, "RYS_META double rys_h[%d] = {0", nmax + 1);
    for (int n = 1; n <= nmax; n++) fprintf(fo, ", %a", hs[n]);
    fprintf(fo, "};\nRYS_META double rys_xmax[%d] = {0", nmax + 1);
    for (int n = 1; n <= nmax; n++) fprintf(fo, ", %a", xas[n]);
    fprintf(fo, "};\nRYS_META int rys_nint[%d] = {0", nmax + 1);
    for (int n = 1; n <= nmax; n++) fprintf(fo, ", %d", nint[n]);
    fprintf(fo, "};\nRYS_META int rys_off[%d] = {0", nmax + 1);
    for (int n = 1; n <= nmax; n++) fprintf(fo, ", %d", off[n]);
    fprintf(fo, "};\n/* Gauss-Hermite limit, node-major: index n*(n-1)/2 + i */\n");
    fprintf(fo, "RYS_META double rys_herm_r[%d] = {", nmax * (nmax + 1) / 2);
    for (int n = 1; n <= nmax; n++)
        for (int i = 0; i < n; i++) fprintf(fo, "%s%a", (n == 1 && i == 0) ? "" : ", ", (double)hr[n][i]);
    fprintf(fo, "};\nRYS_META double rys_herm_w[%d] = {", nmax * (nmax + 1) / 2);
    for (int n = 1; n <= nmax; n++)
        for (int i = 0; i < n; i++) fprintf(fo, "%s%a", (n == 1 && i == 0) ? "" : ", ", (double)hh[n][i]);
    fprintf(fo, "};\n/* compile-time copies of the per-n sizes */\n#ifdef __CUDACC__\n#define RYS_HD __host__ __device__\n"
                "#else\n#define RYS_HD\n#endif\nRYS_HD constexpr int rys_nint_c(int n) { return ");
    for (int n = 1; n <= nmax; n++) fprintf(fo, "n == %d ? %d : ", n, nint[n]);
    fprintf(fo, "0; }\nRYS_HD constexpr int rys_off_c(int n) { return ");
    for (int n = 1; n <= nmax; n++) fprintf(fo, "n == %d ? %d : ", n, off[n]);
    fprintf(fo, "0; }\nRYS_HD constexpr double rys_xmax_c(int n) { return ");
    for (int n = 1; n <= nmax; n++) fprintf(fo, "n == %d ? %a : ", n, xas[n]);
    fprintf(fo, "0.; }\n");
    fprintf(fo, "#ifdef RYS_WANT_COEF\nstatic const double rys_coef[%d] = {\n", off[nmax + 1]);
    for (int n = 1; n <= nmax; n++) {
        size_t cnt = (size_t)nint[n] * 2 * n * NC;
        for (size_t k = 0; k < cnt; k++)
            fprintf(fo, "%a,%s", tables[n][k], (k % 4 == 3) ? "\n" : " ");
    }
    fprintf(fo, "};\n#endif\n");
    fclose(fo);
    return 0;
}
