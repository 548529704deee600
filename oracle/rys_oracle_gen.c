/*
 * ORACLE (test infrastructure only): generator of the oracle's own Rys
 * quadrature tables.  It deliberately uses a different route from the
 * product's generator so the two cross-check each other:
 *
 *   - the Rys measure  int_0^1 f(t^2) exp(-x t^2) dt  is discretised by a
 *     composite Gauss-Legendre rule in t (20 panels x 30 points, nodes found
 *     by Newton iteration on P_30 in __float128);
 *   - recurrence coefficients come from the discretised Stieltjes procedure;
 *   - nodes and weights come from the implicit QL algorithm (Wilkinson
 *     shifts) on the Jacobi matrix, weights = mu0 * (first eigenvector
 *     component)^2 (Golub-Welsch);
 *   - fits: Chebyshev series of 16 terms on intervals of width 2.5;
 *   - x >= X_n: the 2n-point Gauss-Hermite limit (same mathematics as the
 *     reference's large-x branch, cuobc/lib/gint/rys_roots.cu:1278-1295),
 *     with X_n = 40 + 6n.
 *
 * The reference's own tables (cuobc/lib/gint/rys_xw.cuh) are not used.
 * Usage: rys_oracle_gen <nmax> <out.h>
 */
#include <math.h>
#include <quadmath.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef __float128 qf;
#define OC 16
#define OH 2.5
#define NPAN 20
#define NGL 30
#define NMAXO 13

static qf gl_t[NGL], gl_w[NGL];

static void gauss_legendre(void) {
    for (int i = 0; i < NGL; i++) {
        qf z = cosq(M_PIq * (i + 0.75Q) / (NGL + 0.5Q)), pp = 0;
        for (int it = 0; it < 100; it++) {
            qf p1 = 1, p2 = 0;
            for (int j = 0; j < NGL; j++) {
                qf p3 = p2;
                p2 = p1;
                p1 = ((2 * j + 1) * z * p2 - j * p3) / (j + 1);
            }
            pp = NGL * (z * p1 - p2) / (z * z - 1);
            qf z1 = z;
            z = z1 - p1 / pp;
            if (fabsq(z - z1) < 1e-33Q) break;
        }
        gl_t[i] = z;
        gl_w[i] = 2 / ((1 - z * z) * pp * pp);
    }
}

/* implicit QL on a symmetric tridiagonal matrix; d: diagonal (-> eigenvalues),
 * e: sub-diagonal e[1..n-1]; z: first components of eigenvectors */
static void ql_implicit(int n, qf *d, qf *e, qf *z) {
    static qf v[2 * NMAXO][2 * NMAXO];
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) v[i][j] = (i == j);
    for (int i = 1; i < n; i++) e[i - 1] = e[i];
    e[n - 1] = 0;
    for (int l = 0; l < n; l++) {
        int iter = 0, m;
        do {
            for (m = l; m < n - 1; m++) {
                qf dd = fabsq(d[m]) + fabsq(d[m + 1]);
                if (fabsq(e[m]) <= 1e-33Q * dd) break;
            }
            if (m != l) {
                if (iter++ == 200) break;
                qf g = (d[l + 1] - d[l]) / (2 * e[l]);
                qf r = hypotq(g, 1);
                g = d[m] - d[l] + e[l] / (g + (g >= 0 ? fabsq(r) : -fabsq(r)));
                qf s = 1, c = 1, p = 0;
                int i;
                for (i = m - 1; i >= l; i--) {
                    qf f = s * e[i], b = c * e[i];
                    r = hypotq(f, g);
                    e[i + 1] = r;
                    if (r == 0) {
                        d[i + 1] -= p;
                        e[m] = 0;
                        break;
                    }
                    s = f / r;
                    c = g / r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2 * c * b;
                    p = s * r;
                    d[i + 1] = g + p;
                    g = c * r - b;
                    for (int k = 0; k < n; k++) {
                        f = v[k][i + 1];
                        v[k][i + 1] = s * v[k][i] + c * f;
                        v[k][i] = c * v[k][i] - s * f;
                    }
                }
                if (r == 0 && i >= l) continue;
                d[l] -= p;
                e[l] = g;
                e[m] = 0;
            }
        } while (m != l);
    }
    /* sort ascending */
    for (int i = 0; i < n; i++) z[i] = v[0][i];
    for (int i = 0; i < n - 1; i++)
        for (int j = i + 1; j < n; j++)
            if (d[j] < d[i]) {
                qf t = d[i]; d[i] = d[j]; d[j] = t;
                t = z[i]; z[i] = z[j]; z[j] = t;
            }
}

static void rys_stieltjes(int n, qf x, qf *s, qf *w) {
    static qf tau[NPAN * NGL], om[NPAN * NGL];
    int np = NPAN * NGL;
    for (int p = 0; p < NPAN; p++)
        for (int i = 0; i < NGL; i++) {
            qf a = (qf)p / NPAN, b = (qf)(p + 1) / NPAN;
            qf t = (a + b) / 2 + (b - a) / 2 * gl_t[i];
            tau[p * NGL + i] = t * t;
            om[p * NGL + i] = (b - a) / 2 * gl_w[i] * expq(-x * t * t);
        }
    static qf p0[NPAN * NGL], p1[NPAN * NGL];
    qf a[NMAXO], b[NMAXO], nrm_prev = 0;
    for (int j = 0; j < np; j++) { p0[j] = 0; p1[j] = 1; }
    for (int k = 0; k < n; k++) {
        qf nrm = 0, num = 0;
        for (int j = 0; j < np; j++) {
            nrm += om[j] * p1[j] * p1[j];
            num += om[j] * tau[j] * p1[j] * p1[j];
        }
        a[k] = num / nrm;
        b[k] = (k == 0) ? nrm : nrm / nrm_prev;
        nrm_prev = nrm;
        for (int j = 0; j < np; j++) {
            qf pn = (tau[j] - a[k]) * p1[j] - (k ? b[k] : 0) * p0[j];
            p0[j] = p1[j];
            p1[j] = pn;
        }
    }
    qf d[NMAXO], e[NMAXO], z[NMAXO];
    for (int k = 0; k < n; k++) { d[k] = a[k]; e[k] = k ? sqrtq(b[k]) : 0; }
    ql_implicit(n, d, e, z);
    for (int i = 0; i < n; i++) { s[i] = d[i]; w[i] = b[0] * z[i] * z[i]; }
}

static void hermite_limit(int n, qf *r, qf *hw) {
    int m = 2 * n;
    qf d[2 * NMAXO], e[2 * NMAXO], z[2 * NMAXO];
    for (int k = 0; k < m; k++) { d[k] = 0; e[k] = k ? sqrtq(k / 2.0Q) : 0; }
    ql_implicit(m, d, e, z);
    for (int i = 0; i < n; i++) {
        r[i] = d[n + i] * d[n + i];
        hw[i] = sqrtq(M_PIq) * z[n + i] * z[n + i];
    }
}

int main(int argc, char **argv) {
    if (argc < 3) return 2;
    int nmax = atoi(argv[1]);
    if (nmax < 1 || nmax > NMAXO) return 2;
    gauss_legendre();
    FILE *fo = fopen(argv[2], "w");
    if (!fo) return 1;
    fprintf(fo, "/* generated by rys_oracle_gen.c (oracle tables) */\n");
    fprintf(fo, "#define ORYS_NC %d\n#define ORYS_H %a\n#define ORYS_NMAX %d\n", OC, OH, nmax);
    int off = 0;
    int offs[16], nints[16];
    double xmax[16];
    fprintf(fo, "static const double orys_coef[] = {\n");
    for (int n = 1; n <= nmax; n++) {
        xmax[n] = 40 + 6 * n;
        int m = (int)ceil(xmax[n] / OH);
        xmax[n] = m * OH;
        offs[n] = off;
        nints[n] = m;
        for (int k = 0; k < m; k++) {
            qf vals[OC][2 * NMAXO];
            for (int j = 0; j < OC; j++) {
                qf t = cosq(M_PIq * (j + 0.5Q) / OC);
                qf x = k * (qf)OH + (qf)OH / 2 * (1 + t);
                qf s[NMAXO], w[NMAXO];
                rys_stieltjes(n, x, s, w);
                for (int i = 0; i < n; i++) { vals[j][i] = s[i]; vals[j][n + i] = w[i]; }
            }
            for (int f = 0; f < 2 * n; f++)
                for (int c = 0; c < OC; c++) {
                    qf acc = 0;
                    for (int j = 0; j < OC; j++) acc += vals[j][f] * cosq(M_PIq * c * (j + 0.5Q) / OC);
                    acc *= 2.0Q / OC;
                    if (c == 0) acc /= 2;
                    fprintf(fo, "%a,%s", (double)acc, (c % 4 == 3) ? "\n" : " ");
                }
        }
        off += m * 2 * n * OC;
    }
    fprintf(fo, "0};\nstatic const int orys_off[] = {0");
    for (int n = 1; n <= nmax; n++) fprintf(fo, ", %d", offs[n]);
    fprintf(fo, "};\nstatic const int orys_nint[] = {0");
    for (int n = 1; n <= nmax; n++) fprintf(fo, ", %d", nints[n]);
    fprintf(fo, "};\nstatic const double orys_xmax[] = {0");
    for (int n = 1; n <= nmax; n++) fprintf(fo, ", %a", xmax[n]);
    fprintf(fo, "};\nstatic const double orys_hr[] = {0");
    for (int n = 1; n <= nmax; n++) {
        qf r[NMAXO], hw[NMAXO];
        hermite_limit(n, r, hw);
        for (int i = 0; i < n; i++) fprintf(fo, ", %a", (double)r[i]);
    }
    fprintf(fo, "};\nstatic const double orys_hw[] = {0");
    for (int n = 1; n <= nmax; n++) {
        qf r[NMAXO], hw[NMAXO];
        hermite_limit(n, r, hw);
        for (int i = 0; i < n; i++) fprintf(fo, ", %a", (double)hw[i]);
    }
    fprintf(fo, "};\n");
    fclose(fo);
    return 0;
}
