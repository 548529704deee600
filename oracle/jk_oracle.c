/*
 * ORACLE -- test infrastructure only.  A plain CPU restatement of the
 * reference's direct-SCF J/K path (ByteQC cuobc get_jk).  Only tests/,
 * __graft_entry__.smoke() and bench.py's CPU-baseline leg load this library;
 * the product never does.
 *
 * What is restated, with the reference lines it follows:
 *   - primitive-pair data a12, e12 (s/p common factors, diagonal-pair
 *     factor), x12/y12/z12: cuobc/lib/gint/pair_data.c:83-141;
 *   - nroots = (li+lj+lk+ll)/2 + 1 and fac = 2 pi^3 / sqrt(pi):
 *     cuobc/lib/gint/g2e.c:30-45;
 *   - the Rys 2D recursion (VRR in n and m with b00, b10, b01, c00, c0p,
 *     then HRR i->j and k->l): cuobc/lib/gvhf/g2e.cu:32-166; x seeded with
 *     the quartet norm, y with e_ij e_kl / (sqrt(a_ij+a_kl) a_ij a_kl),
 *     z with the weight (g2e.cu:44-54, 87, 227, 367);
 *   - the quartet norm halved when bas_ij == bas_kl and the bas_ij < bas_kl
 *     skip: cuobc/lib/gvhf/g2e.cu:1021-1029;
 *   - the six J/K updates of one quartet, written through the reference's
 *     column-major view v[i + nao*j]: cuobc/lib/gvhf/contract_jk.cu:225-316;
 *   - the bin loop: kl bin b pairs with ij bins [0, nbins-b):
 *     cuobc/lib/gvhf/nr_jk_driver.cu:252-280;
 *   - the Schwarz matrix q[ish,jsh] = sqrt(max |(ij|ij)|) over the Cartesian
 *     functions of the pair, as PySCF's CVHFsetnr_direct_scf computes it for
 *     the reference (cuobc/scf/hf.py:341; PySCF 2.5.0, not vendored).
 *
 * Rys nodes and weights come from the oracle's own tables (rys_oracle_gen.c,
 * a different algorithm from the product's generator).
 *
 * Parallelism: OpenMP over the ij shell pairs of a task; every thread owns
 * private J/K buffers that are summed in thread order, so the result is
 * deterministic for a fixed thread count.
 */
#include <math.h>
#include <omp.h>
#include <stdlib.h>
#include <string.h>

#include "_build/rys_oracle_table.h"

#define ATM_SLOTS 6
#define PTR_COORD 1
#define BAS_SLOTS 8
#define ATOM_OF 0
#define ANG_OF 1
#define NPRIM_OF 2
#define PTR_EXP 5
#define PTR_COEFF 6
#define LMAX 6
#define NF_MAX 28

static double common_fac_sp(int l) {
    if (l == 0) return 0.282094791773878143;
    if (l == 1) return 0.488602511902919921;
    return 1.0;
}

static double cheb(const double *c, double t) {
    double b1 = 0, b2 = 0;
    for (int k = ORYS_NC - 1; k >= 1; k--) {
        double b0 = 2 * t * b1 - b2 + c[k];
        b2 = b1;
        b1 = b0;
    }
    return t * b1 - b2 + c[0];
}

/* Rys nodes s = t^2 and weights for n roots at x */
int oracle_rys_roots(int n, double x, double *s, double *w) {
    if (n < 1 || n > ORYS_NMAX || !(x >= 0)) return 1;
    if (x >= orys_xmax[n]) {
        int base = 1 + n * (n - 1) / 2;
        double sx = sqrt(x);
        for (int i = 0; i < n; i++) {
            s[i] = orys_hr[base + i] / x;
            w[i] = orys_hw[base + i] / sx;
        }
        return 0;
    }
    int m = (int)(x / ORYS_H);
    double t = (x - (m + 0.5) * ORYS_H) / (0.5 * ORYS_H);
    const double *c = orys_coef + orys_off[n] + (size_t)m * 2 * n * ORYS_NC;
    for (int i = 0; i < n; i++) {
        s[i] = cheb(c + i * ORYS_NC, t);
        w[i] = cheb(c + (n + i) * ORYS_NC, t);
    }
    return 0;
}

/* ---- basis helpers --------------------------------------------------- */
typedef struct {
    const int *atm, *bas;
    const double *env;
    int nbas;
} basis_t;

static const double *shell_center(const basis_t *b, int ish) {
    int ia = b->bas[ish * BAS_SLOTS + ATOM_OF];
    return b->env + b->atm[ia * ATM_SLOTS + PTR_COORD];
}

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

/* Cartesian exponents in libcint order */
static void cart_list(int l, int *lx, int *ly, int *lz) {
    int n = 0;
    for (int a = l; a >= 0; a--)
        for (int b = l - a; b >= 0; b--) {
            lx[n] = a;
            ly[n] = b;
            lz[n] = l - a - b;
            n++;
        }
}

/* one primitive pair: a12, e12, P (pair_data.c:108-139) */
static void prim_pair(const basis_t *b, int ish, int jsh, int ip, int jp, double diag_fac,
                      double *aij, double *eij, double *P) {
    const double *ri = shell_center(b, ish), *rj = shell_center(b, jsh);
    double ai = b->env[b->bas[ish * BAS_SLOTS + PTR_EXP] + ip];
    double aj = b->env[b->bas[jsh * BAS_SLOTS + PTR_EXP] + jp];
    double ci = b->env[b->bas[ish * BAS_SLOTS + PTR_COEFF] + ip];
    double cj = b->env[b->bas[jsh * BAS_SLOTS + PTR_COEFF] + jp];
    int li = b->bas[ish * BAS_SLOTS + ANG_OF], lj = b->bas[jsh * BAS_SLOTS + ANG_OF];
    double dx = ri[0] - rj[0], dy = ri[1] - rj[1], dz = ri[2] - rj[2];
    double r2 = dx * dx + dy * dy + dz * dz;
    double a = ai + aj;
    *aij = a;
    *eij = common_fac_sp(li) * common_fac_sp(lj) * ci * cj * exp(-r2 * ai * aj / a);
    if (ish == jsh) *eij *= diag_fac;
    for (int d = 0; d < 3; d++) P[d] = (ai * ri[d] + aj * rj[d]) / a;
}

/*
 * Contracted Cartesian ERI block out[i + nfi*(j + nfj*(k + nfk*l))] of the
 * shell quartet, times `norm` (the reference seeds its x integrals with
 * fac = 2 pi^3/sqrt(pi), halved when bas_ij == bas_kl), with e12 of the
 * diagonal pairs scaled by diag_fac as in the reference pair cache.
 */
static void eri_quartet(const basis_t *b, int ish, int jsh, int ksh, int lsh, double diag_fac,
                        double norm, double *out) {
    int li = b->bas[ish * BAS_SLOTS + ANG_OF], lj = b->bas[jsh * BAS_SLOTS + ANG_OF];
    int lk = b->bas[ksh * BAS_SLOTS + ANG_OF], ll = b->bas[lsh * BAS_SLOTS + ANG_OF];
    int npi = b->bas[ish * BAS_SLOTS + NPRIM_OF], npj = b->bas[jsh * BAS_SLOTS + NPRIM_OF];
    int npk = b->bas[ksh * BAS_SLOTS + NPRIM_OF], npl = b->bas[lsh * BAS_SLOTS + NPRIM_OF];
    int nfi = ncart(li), nfj = ncart(lj), nfk = ncart(lk), nfl = ncart(ll);
    int nf = nfi * nfj * nfk * nfl;
    int nroots = (li + lj + lk + ll) / 2 + 1;
    int nmax = li + lj, mmax = lk + ll;
    const double *ri = shell_center(b, ish), *rj = shell_center(b, jsh);
    const double *rk = shell_center(b, ksh), *rl = shell_center(b, lsh);
    int ix[NF_MAX], iy[NF_MAX], iz[NF_MAX], jx[NF_MAX], jy[NF_MAX], jz[NF_MAX];
    int kx[NF_MAX], ky[NF_MAX], kz[NF_MAX], lx[NF_MAX], ly[NF_MAX], lz[NF_MAX];
    cart_list(li, ix, iy, iz);
    cart_list(lj, jx, jy, jz);
    cart_list(lk, kx, ky, kz);
    cart_list(ll, lx, ly, lz);
    memset(out, 0, sizeof(double) * nf);
    /* G[axis][n][m] then I[axis][i][j][k][l] */
    double G[3][2 * LMAX + 1][2 * LMAX + 1];
    double I[3][LMAX + 1][LMAX + 1][LMAX + 1][LMAX + 1];
    double Itmp[2 * LMAX + 1][LMAX + 1][2 * LMAX + 1];
    for (int ip = 0; ip < npi; ip++)
        for (int jp = 0; jp < npj; jp++) {
            double aij, eij, P[3];
            prim_pair(b, ish, jsh, ip, jp, diag_fac, &aij, &eij, P);
            for (int kp = 0; kp < npk; kp++)
                for (int lp = 0; lp < npl; lp++) {
                    double akl, ekl, Q[3];
                    prim_pair(b, ksh, lsh, kp, lp, diag_fac, &akl, &ekl, Q);
                    double A = aij, B = akl, AB = A + B;
                    double rho = A * B / AB;
                    double pq2 = 0;
                    for (int d = 0; d < 3; d++) pq2 += (P[d] - Q[d]) * (P[d] - Q[d]);
                    double x = rho * pq2;
                    double rs[16], rw[16];
                    oracle_rys_roots(nroots, x, rs, rw);
                    double seed[3];
                    seed[0] = norm;
                    seed[1] = eij * ekl / (sqrt(AB) * A * B);
                    for (int r = 0; r < nroots; r++) {
                        double s = rs[r];
                        seed[2] = rw[r];
                        double b00 = 0.5 * s / AB;
                        double b10 = 0.5 / A * (1 - B * s / AB);
                        double b01 = 0.5 / B * (1 - A * s / AB);
                        for (int d = 0; d < 3; d++) {
                            double c00 = (P[d] - ri[d]) - B * s / AB * (P[d] - Q[d]);
                            double c0p = (Q[d] - rk[d]) + A * s / AB * (P[d] - Q[d]);
                            /* VRR */
                            G[d][0][0] = seed[d];
                            for (int n = 0; n < nmax; n++)
                                G[d][n + 1][0] = c00 * G[d][n][0] + (n ? n * b10 * G[d][n - 1][0] : 0);
                            for (int m = 0; m < mmax; m++)
                                for (int n = 0; n <= nmax; n++)
                                    G[d][n][m + 1] = c0p * G[d][n][m] + (m ? m * b01 * G[d][n][m - 1] : 0) +
                                                     (n ? n * b00 * G[d][n - 1][m] : 0);
                            /* HRR i -> j: (a, j+1) = (a+1, j) + (Ri - Rj)(a, j) */
                            double dij = ri[d] - rj[d], dkl = rk[d] - rl[d];
                            for (int m = 0; m <= mmax; m++) {
                                for (int a = 0; a <= nmax; a++) Itmp[a][0][m] = G[d][a][m];
                                for (int j = 1; j <= lj; j++)
                                    for (int a = 0; a <= nmax - j; a++)
                                        Itmp[a][j][m] = Itmp[a + 1][j - 1][m] + dij * Itmp[a][j - 1][m];
                            }
                            /* HRR k -> l for every (i, j) */
                            for (int i = 0; i <= li; i++)
                                for (int j = 0; j <= lj; j++) {
                                    double T[2 * LMAX + 1][LMAX + 1];
                                    for (int c = 0; c <= mmax; c++) T[c][0] = Itmp[i][j][c];
                                    for (int l = 1; l <= ll; l++)
                                        for (int c = 0; c <= mmax - l; c++)
                                            T[c][l] = T[c + 1][l - 1] + dkl * T[c][l - 1];
                                    for (int k = 0; k <= lk; k++)
                                        for (int l = 0; l <= ll; l++) I[d][i][j][k][l] = T[k][l];
                                }
                        }
                        for (int l = 0; l < nfl; l++)
                            for (int k = 0; k < nfk; k++)
                                for (int j = 0; j < nfj; j++)
                                    for (int i = 0; i < nfi; i++)
                                        out[i + nfi * (j + nfj * (k + nfk * l))] +=
                                            I[0][ix[i]][jx[j]][kx[k]][lx[l]] *
                                            I[1][iy[i]][jy[j]][ky[k]][ly[l]] *
                                            I[2][iz[i]][jz[j]][kz[k]][lz[l]];
                    }
                }
        }
}

/* Contracted Cartesian ERIs (ij|kl) of one shell quartet in libcint
 * normalisation (no symmetry factors): out[i + nfi*(j + nfj*(k + nfk*l))]. */
void oracle_eri_shells(const int *atm, const int *bas, const double *env, int nbas, int ish, int jsh,
                       int ksh, int lsh, double *out) {
    basis_t b = {atm, bas, env, nbas};
    eri_quartet(&b, ish, jsh, ksh, lsh, 1.0, 2 * M_PI * M_PI * M_PI / sqrt(M_PI), out);
}

/* q[ish*nbas + jsh] = sqrt(max_{i in ish, j in jsh} |(ij|ij)|) */
void oracle_q_cond(const int *atm, const int *bas, const double *env, int nbas, double *q) {
    basis_t b = {atm, bas, env, nbas};
    double fac = 2 * M_PI * M_PI * M_PI / sqrt(M_PI);
#pragma omp parallel
    {
        double *buf = malloc(sizeof(double) * NF_MAX * NF_MAX * NF_MAX * NF_MAX);
#pragma omp for schedule(dynamic, 4)
        for (int ish = 0; ish < nbas; ish++)
            for (int jsh = 0; jsh <= ish; jsh++) {
                int nfi = ncart(bas[ish * BAS_SLOTS + ANG_OF]);
                int nfj = ncart(bas[jsh * BAS_SLOTS + ANG_OF]);
                eri_quartet(&b, ish, jsh, ish, jsh, 1.0, fac, buf);
                double mx = 0;
                for (int j = 0; j < nfj; j++)
                    for (int i = 0; i < nfi; i++) {
                        double v = fabs(buf[i + nfi * (j + nfj * (i + nfi * j))]);
                        if (v > mx) mx = v;
                    }
                q[ish * nbas + jsh] = q[jsh * nbas + ish] = sqrt(mx);
            }
        free(buf);
    }
}

/*
 * One task of the reference get_jk: class pair (cp_ij, cp_kl) with the
 * reference bin offsets (host arrays, nbins+1 entries, local to the class),
 * accumulated into vj/vk (either may be NULL) with the reference's view
 * convention v[i + nao*j].  pair_locs: start of each class in pair2bra/ket.
 * ij_stride > 1 evaluates only the rows ij = ij_offset mod ij_stride (a
 * uniform subsample used to time the CPU baseline on a bounded share of the
 * work); count_only returns the number of quartets without evaluating them.
 * dm: (n_dm, nao, nao) C-order.  Returns the number of contracted quartets
 * evaluated.
 *
 * Between oracle_jk_begin and oracle_jk_end the per-thread accumulators live
 * across calls (allocated and zeroed once, summed into vj/vk once by
 * oracle_jk_end); otherwise every call allocates and reduces its own.
 */
static double *g_vjt = NULL, *g_vkt = NULL;
static size_t g_nn = 0;

int oracle_jk_begin(int nao, int n_dm, int with_j, int with_k) {
    g_nn = (size_t)nao * nao * n_dm;
    int nthreads = omp_get_max_threads();
    g_vjt = with_j ? calloc(g_nn * nthreads, sizeof(double)) : NULL;
    g_vkt = with_k ? calloc(g_nn * nthreads, sizeof(double)) : NULL;
    return ((with_j && !g_vjt) || (with_k && !g_vkt)) ? 1 : 0;
}

void oracle_jk_end(double *vj, double *vk) {
    int nthreads = omp_get_max_threads();
    for (int t = 0; t < nthreads; t++)
        for (size_t x = 0; x < g_nn; x++) {
            if (vj && g_vjt) vj[x] += g_vjt[g_nn * t + x];
            if (vk && g_vkt) vk[x] += g_vkt[g_nn * t + x];
        }
    free(g_vjt);
    free(g_vkt);
    g_vjt = g_vkt = NULL;
    g_nn = 0;
}

long oracle_build_jk(const int *atm, const int *bas, const double *env, int nbas, const int *ao_loc,
                     const int *pair2bra, const int *pair2ket, const int *pair_locs, double diag_fac,
                     const double *dm, int nao, int n_dm, double *vj, double *vk,
                     const int *bins_ij, const int *bins_kl, int nbins, int cp_ij, int cp_kl,
                     int ij_stride, int ij_offset, int count_only) {
    basis_t b = {atm, bas, env, nbas};
    double fac = 2 * M_PI * M_PI * M_PI / sqrt(M_PI);
    long count = 0;
    size_t nn = (size_t)nao * nao * n_dm;
    int nthreads = omp_get_max_threads();
    const int shared_ws = g_nn == nn && (g_vjt || g_vkt);
    double *vjt = (vj && !count_only) ? (shared_ws ? g_vjt : calloc(nn * nthreads, sizeof(double))) : NULL;
    double *vkt = (vk && !count_only) ? (shared_ws ? g_vkt : calloc(nn * nthreads, sizeof(double))) : NULL;
    for (int kl_bin = 0; kl_bin < nbins; kl_bin++) {
        int kl0 = bins_kl[kl_bin], kl1 = bins_kl[kl_bin + 1];
        if (kl1 - kl0 <= 0) continue;
        int ij1 = bins_ij[nbins - kl_bin];
        int ij0 = bins_ij[0];
        if (ij1 - ij0 <= 0) continue;
#pragma omp parallel reduction(+ : count)
        {
            int tid = omp_get_thread_num();
            double *myj = vjt ? vjt + nn * tid : NULL;
            double *myk = vkt ? vkt + nn * tid : NULL;
            double *g = malloc(sizeof(double) * NF_MAX * NF_MAX * NF_MAX * NF_MAX);
            // rows of the (sub)sample; the loop runs over (row, kl) so that a
            // subsample with few rows still uses every thread
            const int rstep = ij_stride > 1 ? ij_stride : 1;
            int r0 = ij0;
            if (rstep > 1) r0 = ij0 + ((ij_offset - ij0 % rstep) % rstep + rstep) % rstep;
            const int nrows = r0 < ij1 ? (ij1 - 1 - r0) / rstep + 1 : 0;
#pragma omp for collapse(2) schedule(dynamic, 64)
            for (int ri = 0; ri < nrows; ri++) {
                for (int tkl = kl0; tkl < kl1; tkl++) {
                    const int tij = r0 + ri * rstep;
                    int bas_ij = pair_locs[cp_ij] + tij;
                    int bas_kl = pair_locs[cp_kl] + tkl;
                    if (bas_ij < bas_kl) continue;
                    if (count_only) {
                        count++;
                        continue;
                    }
                    double norm = fac;
                    if (bas_ij == bas_kl) norm *= .5;
                    int ish = pair2bra[bas_ij], jsh = pair2ket[bas_ij];
                    int ksh = pair2bra[bas_kl], lsh = pair2ket[bas_kl];
                    eri_quartet(&b, ish, jsh, ksh, lsh, diag_fac, norm, g);
                    count++;
                    int i0 = ao_loc[ish], j0 = ao_loc[jsh], k0 = ao_loc[ksh], l0 = ao_loc[lsh];
                    int nfi = ao_loc[ish + 1] - i0, nfj = ao_loc[jsh + 1] - j0;
                    int nfk = ao_loc[ksh + 1] - k0, nfl = ao_loc[lsh + 1] - l0;
                    for (int idm = 0; idm < n_dm; idm++) {
                        const double *D = dm + (size_t)idm * nao * nao;
                        double *J = myj ? myj + (size_t)idm * nao * nao : NULL;
                        double *K = myk ? myk + (size_t)idm * nao * nao : NULL;
                        for (int l = 0; l < nfl; l++)
                            for (int k = 0; k < nfk; k++)
                                for (int j = 0; j < nfj; j++)
                                    for (int i = 0; i < nfi; i++) {
                                        double s = g[i + nfi * (j + nfj * (k + nfk * l))];
                                        int I = i0 + i, Jj = j0 + j, Kk = k0 + k, L = l0 + l;
                                        if (J) {
                                            J[I + (size_t)nao * Jj] += s * D[Kk + (size_t)nao * L];
                                            J[Kk + (size_t)nao * L] += s * D[I + (size_t)nao * Jj];
                                        }
                                        if (K) {
                                            K[I + (size_t)nao * Kk] += s * D[Jj + (size_t)nao * L];
                                            K[I + (size_t)nao * L] += s * D[Jj + (size_t)nao * Kk];
                                            K[Jj + (size_t)nao * Kk] += s * D[I + (size_t)nao * L];
                                            K[Jj + (size_t)nao * L] += s * D[I + (size_t)nao * Kk];
                                        }
                                    }
                    }
                }
            }
            free(g);
        }
    }
    if (!shared_ws) {
        for (int t = 0; t < nthreads; t++)
            for (size_t x = 0; x < nn; x++) {
                if (vjt) vj[x] += vjt[nn * t + x];
                if (vkt) vk[x] += vkt[nn * t + x];
            }
        free(vjt);
        free(vkt);
    }
    return count;
}

/* ---- overlap ---------------------------------------------------------- */
/* Cartesian overlap <i|j> of a basis whose shells carry one contraction
 * each (the decontracted working basis), in libcint's conventions: the
 * env coefficients hold the radial normalisation, the s and p common
 * factors are applied at evaluation time (as for the ERIs above).  1D
 * overlaps by the Obara-Saika recursion on the Gaussian product centre,
 * S(a+1,0) = PA S(a,0) + a/(2g) S(a-1,0), then S(a,b+1) = S(a+1,b) + AB S(a,b).
 * Used to build test densities and to check the normalisation of the
 * contracted spherical basis without the product library.  Returns 1 for a
 * shell with more than one contraction or l > LMAX. */
int oracle_ovlp_cart(const int *atm, const int *bas, const double *env, int nbas, const int *ao_loc,
                     double *out) {
    basis_t b = {atm, bas, env, nbas};
    int nao = ao_loc[nbas];
    for (int s = 0; s < nbas; s++)
        if (bas[s * BAS_SLOTS + 3] != 1 || bas[s * BAS_SLOTS + ANG_OF] > LMAX) return 1;
#pragma omp parallel for schedule(dynamic)
    for (int ish = 0; ish < nbas; ish++) {
        for (int jsh = 0; jsh < nbas; jsh++) {
            int li = bas[ish * BAS_SLOTS + ANG_OF], lj = bas[jsh * BAS_SLOTS + ANG_OF];
            int npi = bas[ish * BAS_SLOTS + NPRIM_OF], npj = bas[jsh * BAS_SLOTS + NPRIM_OF];
            const double *ri = shell_center(&b, ish), *rj = shell_center(&b, jsh);
            const double *ei = env + bas[ish * BAS_SLOTS + PTR_EXP], *ej = env + bas[jsh * BAS_SLOTS + PTR_EXP];
            const double *ci = env + bas[ish * BAS_SLOTS + PTR_COEFF], *cj = env + bas[jsh * BAS_SLOTS + PTR_COEFF];
            int lxi[NF_MAX], lyi[NF_MAX], lzi[NF_MAX], lxj[NF_MAX], lyj[NF_MAX], lzj[NF_MAX];
            cart_list(li, lxi, lyi, lzi);
            cart_list(lj, lxj, lyj, lzj);
            int nfi = ncart(li), nfj = ncart(lj);
            double blk[NF_MAX * NF_MAX];
            memset(blk, 0, sizeof(blk));
            double r2 = 0;
            for (int d = 0; d < 3; d++) r2 += (ri[d] - rj[d]) * (ri[d] - rj[d]);
            for (int ip = 0; ip < npi; ip++)
                for (int jp = 0; jp < npj; jp++) {
                    double a = ei[ip], c = ej[jp], g = a + c;
                    double pref = ci[ip] * cj[jp] * exp(-a * c / g * r2) * pow(M_PI / g, 1.5);
                    double s1[3][2 * LMAX + 2][LMAX + 1];
                    for (int d = 0; d < 3; d++) {
                        double P = (a * ri[d] + c * rj[d]) / g;
                        double PA = P - ri[d], AB = ri[d] - rj[d];
                        double t[2 * LMAX + 2][LMAX + 1];
                        t[0][0] = 1.;
                        for (int x = 0; x < li + lj; x++)
                            t[x + 1][0] = PA * t[x][0] + (x > 0 ? x / (2 * g) * t[x - 1][0] : 0.);
                        for (int y = 0; y < lj; y++)
                            for (int x = 0; x + y + 1 <= li + lj; x++) t[x][y + 1] = t[x + 1][y] + AB * t[x][y];
                        for (int x = 0; x <= li; x++)
                            for (int y = 0; y <= lj; y++) s1[d][x][y] = t[x][y];
                    }
                    for (int i = 0; i < nfi; i++)
                        for (int j = 0; j < nfj; j++)
                            blk[i * nfj + j] += pref * s1[0][lxi[i]][lxj[j]] * s1[1][lyi[i]][lyj[j]] *
                                                s1[2][lzi[i]][lzj[j]];
                }
            double f = common_fac_sp(li) * common_fac_sp(lj);
            for (int i = 0; i < nfi; i++)
                for (int j = 0; j < nfj; j++)
                    out[(size_t)(ao_loc[ish] + i) * nao + ao_loc[jsh] + j] = f * blk[i * nfj + j];
        }
    }
    return 0;
}

/* The primitive-pair table of a pair list in the reference's cache layout
 * (a12 | e12 | x12 | y12 | z12, each n_prim_pairs long, pairs in list order,
 * primitives bra-major; pair_data.c:83-141), from prim_pair above.  Lets the
 * tests compare the oracle's pair data with the reference's own
 * GINTinit_aexyz. */
long oracle_pair_data(const int *atm, const int *bas, const double *env, int nbas, const int *pair2bra,
                      const int *pair2ket, int npairs, double diag_fac, double *out, long cap) {
    basis_t b = {atm, bas, env, nbas};
    long n = 0;
    for (int p = 0; p < npairs; p++)
        n += (long)bas[pair2bra[p] * BAS_SLOTS + NPRIM_OF] * bas[pair2ket[p] * BAS_SLOTS + NPRIM_OF];
    if (n > cap) return -n;
    long c = 0;
    for (int p = 0; p < npairs; p++) {
        int ish = pair2bra[p], jsh = pair2ket[p];
        int npi = bas[ish * BAS_SLOTS + NPRIM_OF], npj = bas[jsh * BAS_SLOTS + NPRIM_OF];
        for (int ip = 0; ip < npi; ip++)
            for (int jp = 0; jp < npj; jp++, c++) {
                double P[3];
                prim_pair(&b, ish, jsh, ip, jp, diag_fac, out + c, out + n + c, P);
                out[2 * n + c] = P[0];
                out[3 * n + c] = P[1];
                out[4 * n + c] = P[2];
            }
    }
    return n;
}
