// C-ABI of the J/K engine (declared in include/byteqc_jk.h): basis setup with
// device-side Schwarz screening, the per-call density screen and quartet
// enumeration on the device, the class launches, and the AO transforms.
#include <cublas_v2.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/byteqc_jk.h"
#include "jk_launch.cuh"
#include "jk_internal.h"

// primitive-pair screen of the thread kernels: exp(-mu r^2) below exp(-60)
// (the default exponent cutoff of libcint's pair data) contributes nothing
#define JK_PRIM_EXPCUT 60.0

// ---------------------------------------------------------------------------
// errors
// ---------------------------------------------------------------------------
static thread_local std::string g_err;

static int set_err(int code, const char* fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

#define CUDA_TRY(x)                                                                               \
    do {                                                                                          \
        cudaError_t e_ = (x);                                                                     \
        if (e_ != cudaSuccess) return set_err(JK_ERR_CUDA, "%s: %s", #x, cudaGetErrorString(e_)); \
    } while (0)

extern "C" const char* jk_last_error(void) { return g_err.c_str(); }

// ---------------------------------------------------------------------------
// launcher tables
// ---------------------------------------------------------------------------
static JKTables g_tabs;
#define g_tab64 g_tabs.t64
#define g_tab32 g_tabs.t32
static std::once_flag g_tab_once;
static void init_tables() {
    std::call_once(g_tab_once, [] {
        JK_REGISTER_ALL();
        jk_register_generic(&g_tabs);
    });
}


static double common_fac_sp(int l) {
    return l == 0 ? 0.282094791773878143 : (l == 1 ? 0.488602511902919921 : 1.0);
}

// ---------------------------------------------------------------------------
// Schwarz matrix on the device: q[i,j] = sqrt(max_{a in i, b in j} |(ab|ab)|)
// over the Cartesian functions of the pair (the quantity PySCF's
// CVHFsetnr_direct_scf gives the reference, cuobc/scf/hf.py:341).
// One thread per shell pair, bra shell of the larger l.
// ---------------------------------------------------------------------------
template <int LI, int LJ>
__global__ void jk_qcond_kernel(const int* __restrict__ pi, const int* __restrict__ pj, int npairs,
                                const int* __restrict__ atm, const int* __restrict__ bas,
                                const double* __restrict__ env, int nbas, double* __restrict__ q,
                                const double* __restrict__ rys) {
    using C = JKClass<LI, LJ, LI, LJ>;
    int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npairs) return;
    int ish = pi[p], jsh = pj[p];
    const double* ri = env + atm[bas[ish * BAS_SLOTS + ATOM_OF] * ATM_SLOTS + PTR_COORD];
    const double* rj = env + atm[bas[jsh * BAS_SLOTS + ATOM_OF] * ATM_SLOTS + PTR_COORD];
    int npi = bas[ish * BAS_SLOTS + NPRIM_OF], npj = bas[jsh * BAS_SLOTS + NPRIM_OF];
    const double* ai = env + bas[ish * BAS_SLOTS + PTR_EXP];
    const double* aj = env + bas[jsh * BAS_SLOTS + PTR_EXP];
    const double* ci = env + bas[ish * BAS_SLOTS + PTR_COEFF];
    const double* cj = env + bas[jsh * BAS_SLOTS + PTR_COEFF];
    double fsp = (LI == 0 ? 0.282094791773878143 : (LI == 1 ? 0.488602511902919921 : 1.0)) *
                 (LJ == 0 ? 0.282094791773878143 : (LJ == 1 ? 0.488602511902919921 : 1.0));
    double r2 = 0;
    for (int d = 0; d < 3; d++) r2 += (ri[d] - rj[d]) * (ri[d] - rj[d]);
    double diag[C::NFI * C::NFJ];
#pragma unroll
    for (int e = 0; e < C::NFI * C::NFJ; e++) diag[e] = 0;
    double r_i[3] = {ri[0], ri[1], ri[2]}, r_j[3] = {rj[0], rj[1], rj[2]};
    for (int ip = 0; ip < npi; ip++)
        for (int jp = 0; jp < npj; jp++) {
            double A = ai[ip] + aj[jp];
            double eij = fsp * ci[ip] * cj[jp] * exp(-r2 * ai[ip] * aj[jp] / A);
            double P[3];
            for (int d = 0; d < 3; d++) P[d] = (ai[ip] * ri[d] + aj[jp] * rj[d]) / A;
            for (int kp = 0; kp < npi; kp++)
                for (int lp = 0; lp < npj; lp++) {
                    double B = ai[kp] + aj[lp];
                    double ekl = fsp * ci[kp] * cj[lp] * exp(-r2 * ai[kp] * aj[lp] / B);
                    JKPrim pr;
                    pr.A = A;
                    pr.B = B;
                    pr.AB = A + B;
                    pr.iA = 1. / A;
                    pr.iB = 1. / B;
                    pr.iAB = 1. / pr.AB;
                    for (int d = 0; d < 3; d++) {
                        pr.P[d] = P[d];
                        pr.Q[d] = (ai[kp] * ri[d] + aj[lp] * rj[d]) / B;
                    }
                    double dx = pr.P[0] - pr.Q[0], dy = pr.P[1] - pr.Q[1], dz = pr.P[2] - pr.Q[2];
                    pr.x = A * B / pr.AB * (dx * dx + dy * dy + dz * dz);
                    pr.sy = eij * ekl / (sqrt(pr.AB) * A * B);
                    for (int r = 0; r < C::NROOTS; r++) {
                        double s, w;
                        rys_root<C::NROOTS>(rys, pr.x, r, s, w);
                        double Ix[C::GS], Iy[C::GS], Iz[C::GS];
                        jk_unit<C, double>(pr, s, w, 0, JK_FAC, r_i, r_j, r_i, r_j, Ix);
                        jk_unit<C, double>(pr, s, w, 1, JK_FAC, r_i, r_j, r_i, r_j, Iy);
                        jk_unit<C, double>(pr, s, w, 2, JK_FAC, r_i, r_j, r_i, r_j, Iz);
#pragma unroll
                        for (int a = 0; a < C::NFI; a++)
#pragma unroll
                            for (int b = 0; b < C::NFJ; b++) {
                                int ox = cart_lx(LI, a) * (C::SI + C::SK) + cart_lx(LJ, b) * (C::SJ + 1);
                                int oy = cart_ly(LI, a) * (C::SI + C::SK) + cart_ly(LJ, b) * (C::SJ + 1);
                                int oz = cart_lz(LI, a) * (C::SI + C::SK) + cart_lz(LJ, b) * (C::SJ + 1);
                                diag[a * C::NFJ + b] += Ix[ox] * Iy[oy] * Iz[oz];
                            }
                    }
                }
        }
    double mx = 0;
#pragma unroll
    for (int e = 0; e < C::NFI * C::NFJ; e++) mx = fmax(mx, fabs(diag[e]));
    double v = sqrt(mx);
    q[(size_t)ish * nbas + jsh] = v;
    q[(size_t)jsh * nbas + ish] = v;
}

// Schwarz diagonal of pairs with a shell above f (jk_generic.cu); lmax is
// the larger l of the pairs in the list
void jk_qcond_generic(const int* pi, const int* pj, int n, const int* atm, const int* bas, const double* env,
                      int nbas, double* q, const double* rys, int lmax, cudaStream_t st);

typedef void (*qcond_fn)(const int*, const int*, int, const int*, const int*, const double*, int, double*,
                         const double*, cudaStream_t);
template <int LI, int LJ>
static void qcond_launch(const int* pi, const int* pj, int n, const int* atm, const int* bas, const double* env,
                         int nbas, double* q, const double* rys, cudaStream_t st) {
    if (n > 0) jk_qcond_kernel<LI, LJ><<<(n + 63) / 64, 64, 0, st>>>(pi, pj, n, atm, bas, env, nbas, q, rys);
}
static qcond_fn g_qcond[4][4] = {
    {qcond_launch<0, 0>, nullptr, nullptr, nullptr},
    {qcond_launch<1, 0>, qcond_launch<1, 1>, nullptr, nullptr},
    {qcond_launch<2, 0>, qcond_launch<2, 1>, qcond_launch<2, 2>, nullptr},
    {qcond_launch<3, 0>, qcond_launch<3, 1>, qcond_launch<3, 2>, qcond_launch<3, 3>},
};

// ---------------------------------------------------------------------------
// per-call kernels: density condensation and quartet screening
// ---------------------------------------------------------------------------
// dm_cond[gi, gj] = max over the dms of max |D[p, q]|, p in group gi, q in gj
// (lib.condense('absmax') over the group AO boundaries, cuobc/scf/hf.py:104-107)
__global__ void jk_dm_cond_kernel(const double* __restrict__ dm, int nao, int n_dm, const int* __restrict__ gao,
                                  int ngroups, double* __restrict__ out) {
    int gi = blockIdx.x, gj = blockIdx.y;
    int p0 = gao[gi], p1 = gao[gi + 1], q0 = gao[gj], q1 = gao[gj + 1];
    int np = p1 - p0, nq = q1 - q0;
    double mx = 0;
    long long n = (long long)np * nq * n_dm;
    for (long long e = threadIdx.x; e < n; e += blockDim.x) {
        int idm = (int)(e / ((long long)np * nq));
        int rem = (int)(e - (long long)idm * np * nq);
        int p = p0 + rem / nq, qq = q0 + rem % nq;
        mx = fmax(mx, fabs(dm[(size_t)idm * nao * nao + (size_t)p * nao + qq]));
    }
    __shared__ double red[256];
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) out[gi * ngroups + gj] = red[0];
}


// Block-wide inclusive scan of two counts (256 threads), with running carries.
__device__ __forceinline__ void jk_block_scan2(long long a, long long b, long long& ia, long long& ib,
                                               long long* wa, long long* wb, long long& carry_a,
                                               long long& carry_b) {
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 1; o < 32; o <<= 1) {
        long long ya = __shfl_up_sync(0xffffffffu, a, o), yb = __shfl_up_sync(0xffffffffu, b, o);
        if (lane >= o) {
            a += ya;
            b += yb;
        }
    }
    if (lane == 31) {
        wa[warp] = a;
        wb[warp] = b;
    }
    __syncthreads();
    if (warp == 0) {
        long long x = (lane < (int)(blockDim.x >> 5)) ? wa[lane] : 0;
        long long y = (lane < (int)(blockDim.x >> 5)) ? wb[lane] : 0;
        for (int o = 1; o < 32; o <<= 1) {
            long long u = __shfl_up_sync(0xffffffffu, x, o), v = __shfl_up_sync(0xffffffffu, y, o);
            if (lane >= o) {
                x += u;
                y += v;
            }
        }
        wa[lane] = x;
        wb[lane] = y;
    }
    __syncthreads();
    ia = a + (warp ? wa[warp - 1] : 0) + carry_a;
    ib = b + (warp ? wb[warp - 1] : 0) + carry_b;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) {
        carry_a = ia;
        carry_b = ib;
    }
    __syncthreads();
}

// max over the six group pairs of a class quartet of the condensed density
__device__ __forceinline__ double jk_cq_sub(const double* c, int ngroups, int gi, int gj, int gk, int gl) {
    return fmax(fmax(fmax(c[gi * ngroups + gj], c[gk * ngroups + gl]), fmax(c[gi * ngroups + gk], c[gj * ngroups + gk])),
                fmax(c[gi * ngroups + gl], c[gj * ngroups + gl]));
}

// One block (256 threads) per class quartet.  Reproduces the reference's
// screening decision per contracted quartet (cuobc/scf/hf.py:136-145,
// 567-578 and cuobc/lib/gvhf/nr_jk_driver.cu:252-280):
//   skip the class quartet if prescreen and max(dm_cond over its 6 group
//   pairs) < tol; else with scale = nbins / log(min(tol/sub, 0.1)) and
//   s = floor(scale * log_q), keep (ij, kl) iff s_ij + s_kl < nbins (and
//   kl <= ij inside a diagonal class quartet).
// Because log_q is sorted descending inside a class, the kept kl of a row
// form a prefix; its length is found by binary search and prefix-summed.
// Mixed precision (fp32_cutoff > 0): the kept prefix of a row splits again
// at the bound q_ij q_kl sub = fp32_cutoff (unclipped log q); the leading
// part (larger bounds) runs in FP64, the tail in FP32.  qoff counts the FP64
// part, qoff32 the FP32 part, whose first column per row is klb[ij].
__global__ void jk_screen_kernel(const JKScreenCQ* __restrict__ cqs, double tol, int nbins, int prescreen,
                                 double fp32_cutoff) {
    const JKScreenCQ cq = cqs[blockIdx.x];
    long long* qoff = cq.qoff;
    long long* qoff32 = cq.qoff32;
    int* klb = cq.klb;
    const double* c = cq.dm_cond;
    const int ngroups = cq.ngroups;
    const double sub = jk_cq_sub(c, ngroups, cq.gi, cq.gj, cq.gk, cq.gl);
    bool skip = prescreen && sub < tol;
    double cutoff = tol / sub;
    double scale = nbins / log(fmin(cutoff, 0.1));
    const bool mixed = fp32_cutoff > 0;
    const double log_thr = mixed ? log(fp32_cutoff / sub) : 0.;  // q_ij q_kl >= fp32_cutoff / sub
    const double* lq_ij = cq.lq_ij;
    const double* lq_kl = cq.lq_kl;
    const double* rq_ij = cq.rq_ij;
    const double* rq_kl = cq.rq_kl;
    bool diag = cq.cp_ij == cq.cp_kl;
    __shared__ long long carry, carry32;
    __shared__ long long wsum[32], wsum32[32];
    if (threadIdx.x == 0) {
        carry = carry32 = 0;
        qoff[0] = 0;
        qoff32[0] = 0;
    }
    __syncthreads();
    for (int base = 0; base < cq.n_ij; base += blockDim.x) {
        int ij = base + threadIdx.x;
        long long cnt = 0, c64 = 0;
        if (!skip && ij < cq.n_ij) {
            int sij = (int)floor(scale * lq_ij[ij]);
            if (sij < nbins) {
                int b = nbins - sij;
                // count kl with floor(scale * lq_kl) < b (non-decreasing in kl)
                int lo = 0, hi = cq.n_kl;
                while (lo < hi) {
                    int mid = (lo + hi) >> 1;
                    if ((int)floor(scale * lq_kl[mid]) < b) lo = mid + 1; else hi = mid;
                }
                cnt = lo;
                if (diag && cnt > ij + 1) cnt = ij + 1;
            }
        }
        c64 = cnt;
        if (mixed && cnt > 0) {
            // kl with rq_ij + rq_kl >= log_thr (non-increasing in kl)
            double need = log_thr - rq_ij[ij];
            int lo = 0, hi = (int)cnt;
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (rq_kl[mid] >= need) lo = mid + 1; else hi = mid;
            }
            c64 = lo;
        }
        if (ij < cq.n_ij) klb[ij] = (int)c64;
        long long i64, i32;
        jk_block_scan2(c64, cnt - c64, i64, i32, wsum, wsum32, carry, carry32);
        if (ij < cq.n_ij) {
            qoff[ij + 1] = i64;
            qoff32[ij + 1] = i32;
        }
    }
    if (threadIdx.x == 0) {
        cq.task0[0] = 0;
        cq.task0[1] = carry;
        cq.task032[0] = 0;
        cq.task032[1] = carry32;
    }
}

// Pair-packed J side of jk_build.  mode 0: gather the density blocks of
// every pair into dp (element c of pair p of class k at off_k + c*np_k + p,
// one copy per density); mode 1: add the packed J accumulators jp into vj.
// Every (pair, component) is a distinct element of D and of vj.
__device__ __forceinline__ void jk_pack_body(const JKPackCls* __restrict__ cls, int ncls, long long total,
                                             const int* __restrict__ pair2bra, const int* __restrict__ pair2ket,
                                             const int* __restrict__ ao_loc, const double* __restrict__ dm, int nao,
                                             int n_dm, double* __restrict__ dp, const double* __restrict__ jp,
                                             double* __restrict__ vj, int mode) {
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
         t += (long long)gridDim.x * blockDim.x) {
        int lo = 0, hi = ncls - 1;
        while (lo < hi) {
            int mid = (lo + hi + 1) >> 1;
            if (cls[mid].off <= t) lo = mid; else hi = mid - 1;
        }
        const JKPackCls k = cls[lo];
        const long long local = t - k.off;
        const int comp = (int)(local / k.np), p = (int)(local - (long long)comp * k.np);
        const int a = comp / k.nfj, bb = comp - a * k.nfj;
        const int pair = k.pair0 + p;
        const size_t e = (size_t)(ao_loc[pair2bra[pair]] + a) + (size_t)nao * (ao_loc[pair2ket[pair]] + bb);
        for (int m = 0; m < n_dm; m++) {
            const size_t mo = (size_t)m * nao * nao;
            if (mode == 0) dp[m * total + t] = dm[mo + e];
            else vj[mo + e] += jp[m * total + t];
        }
    }
}

__global__ void jk_pack_kernel(const JKPackCls* __restrict__ cls, int ncls, long long total,
                               const int* __restrict__ pair2bra, const int* __restrict__ pair2ket,
                               const int* __restrict__ ao_loc, const double* __restrict__ dm, int nao, int n_dm,
                               double* __restrict__ dp, const double* __restrict__ jp, double* __restrict__ vj,
                               int mode) {
    jk_pack_body(cls, ncls, total, pair2bra, pair2ket, ao_loc, dm, nao, n_dm, dp, jp, vj, mode);
}

// one molecule per blockIdx.y
__global__ void jk_pack_batch_kernel(const JKPackMol* __restrict__ mols, int mode) {
    const JKPackMol m = mols[blockIdx.y];
    if (m.total <= 0) return;
    jk_pack_body(m.cls, m.ncls, m.total, m.pair2bra, m.pair2ket, m.ao_loc, m.dm, m.nao, m.n_dm, m.dp, m.jp, m.vj,
                 mode);
}

// J = 2 (V + V^T), K = V + V^T in place on the working-basis buffers, where
// V[i, j] = mem[i + nao j]; out_rm[p, q] = fac (mem[p nao + q] + mem[q nao + p])
__global__ void jk_symmetrize_kernel(const double* __restrict__ in, double* __restrict__ out, int nao, int n_dm,
                                     double fac) {
    long long n = (long long)nao * nao * n_dm;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n; e += (long long)gridDim.x * blockDim.x) {
        long long m = e / ((long long)nao * nao);
        long long r = e - m * nao * nao;
        int p = (int)(r / nao), q = (int)(r % nao);
        const double* b = in + m * nao * nao;
        out[e] = fac * (b[(size_t)p * nao + q] + b[(size_t)q * nao + p]);
    }
}

// ---------------------------------------------------------------------------
// basis object
// ---------------------------------------------------------------------------

static void free_basis(jk_basis* b) {
    if (!b) return;
    cudaFree(b->d_atm);
    cudaFree(b->d_bas);
    cudaFree(b->d_ao_loc);
    cudaFree(b->d_group_ao);
    cudaFree(b->d_env);
    cudaFree(b->d_bas_x);
    cudaFree(b->d_qcond);
    cudaFree(b->d_pair2bra);
    cudaFree(b->d_pair2ket);
    cudaFree(b->d_log_q);
    cudaFree(b->d_log_q_raw);
    cudaFree(b->d_qoff32);
    cudaFree(b->d_task032);
    cudaFree(b->d_klb);
    cudaFree(b->d_prim);
    cudaFree(b->d_primf);
    cudaFree(b->d_cq);
    cudaFree(b->d_qoff);
    cudaFree(b->d_task0);
    cudaFree(b->d_dm_cond);
    cudaFree(b->d_qoff1);
    cudaFree(b->d_task01);
    cudaFree(b->d_work);
    cudaFree(b->d_pack);
    cudaFree(b->d_pgeo);
    cudaFree(b->d_pnp);
    cudaFree(b->d_pao);
    b->fan.destroy();
    cudaFree(b->d_pk);
    if (b->blas) cublasDestroy(b->blas);
    delete b;
}

template <typename T>
static cudaError_t upload(T** dst, const T* src, size_t n) {
    cudaError_t e = cudaMalloc((void**)dst, sizeof(T) * (n ? n : 1));
    if (e != cudaSuccess) return e;
    if (n) e = cudaMemcpy(*dst, src, sizeof(T) * n, cudaMemcpyHostToDevice);
    return e;
}

extern "C" int jk_rys_table_uniform(void);
extern "C" const double* jk_rys_coef_host(long long* count);

// Rys coefficient table in global memory, one copy per device, kept until exit
static std::mutex g_rys_mu;
static double* g_rys_dev[64];
static int rys_table_device(const double** out) {
    int dev;
    CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) return set_err(JK_ERR_ARG, "device ordinal %d out of range", dev);
    std::lock_guard<std::mutex> lk(g_rys_mu);
    if (!g_rys_dev[dev]) {
        long long n;
        const double* h = jk_rys_coef_host(&n);
        double* d;
        CUDA_TRY(cudaMalloc(&d, sizeof(double) * n));
        cudaError_t e = cudaMemcpy(d, h, sizeof(double) * n, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(d);
            CUDA_TRY(e);
        }
        g_rys_dev[dev] = d;
    }
    *out = g_rys_dev[dev];
    return JK_OK;
}

static int create_impl(const int* atm, int natm, const int* bas, int nbas, const double* env, int nenv,
                       const int* group_off, int ngroups, double cutoff, int diag_block_with_triu, jk_basis* b) {
    init_tables();
    if (!jk_rys_table_uniform()) return set_err(JK_ERR_ARG, "Rys tables must use intervals of width 2");
    {
        int rc = rys_table_device(&b->rys);
        if (rc) return rc;
    }
    CUDA_TRY(cudaGetDevice(&b->device));
    CUDA_TRY(cudaDeviceGetAttribute(&b->nsm, cudaDevAttrMultiProcessorCount, b->device));
    b->natm = natm;
    b->nbas = nbas;
    b->ngroups = ngroups;
    b->cutoff = cutoff;
    b->diag_fac = diag_block_with_triu ? 1.0 : 0.5;
    // shells must be sorted into groups of equal (l, nprim), one contraction each
    b->h_group_off.assign(group_off, group_off + ngroups + 1);
    if (b->h_group_off[0] != 0 || b->h_group_off[ngroups] != nbas)
        return set_err(JK_ERR_ARG, "group offsets must span 0..nbas");
    b->h_ao_loc.resize(nbas + 1);
    b->h_ao_loc[0] = 0;
    for (int i = 0; i < nbas; i++) {
        int l = bas[i * BAS_SLOTS + ANG_OF];
        if (l < 0 || l > JK_LMAX_ALL)
            return set_err(JK_ERR_UNSUPPORTED, "shell %d has l=%d; this engine handles l <= %d", i, l, JK_LMAX_ALL);
        if (bas[i * BAS_SLOTS + NCTR_OF] != 1)
            return set_err(JK_ERR_ARG, "shell %d: generally contracted shells must be split first", i);
        b->h_ao_loc[i + 1] = b->h_ao_loc[i] + (l + 1) * (l + 2) / 2;
    }
    b->nao = b->h_ao_loc[nbas];
    for (int g = 0; g < ngroups; g++) {
        int s0 = group_off[g], s1 = group_off[g + 1];
        if (s1 <= s0) return set_err(JK_ERR_ARG, "empty group %d", g);
        int l = bas[s0 * BAS_SLOTS + ANG_OF], np = bas[s0 * BAS_SLOTS + NPRIM_OF];
        for (int s = s0; s < s1; s++)
            if (bas[s * BAS_SLOTS + ANG_OF] != l || bas[s * BAS_SLOTS + NPRIM_OF] != np)
                return set_err(JK_ERR_ARG, "group %d mixes (l, nprim)", g);
        // groups may come in any l order (the density-fitting basis of
        // int3c concatenates molecule, exponent-0 shell and auxiliary
        // basis); the J/K class launches exist for classes whose bra and
        // ket are ordered by l, others report JK_ERR_UNSUPPORTED at build
        b->h_group_l.push_back(l);
        b->h_group_nprim.push_back(np);
    }
    // device copies of the basis
    CUDA_TRY(upload(&b->d_atm, atm, (size_t)natm * ATM_SLOTS));
    CUDA_TRY(upload(&b->d_bas, bas, (size_t)nbas * BAS_SLOTS));
    CUDA_TRY(upload(&b->d_env, env, (size_t)nenv));
    CUDA_TRY(upload(&b->d_ao_loc, b->h_ao_loc.data(), b->h_ao_loc.size()));
    std::vector<int> gao(ngroups + 1);
    for (int g = 0; g <= ngroups; g++) gao[g] = b->h_ao_loc[group_off[g]];
    CUDA_TRY(upload(&b->d_group_ao, gao.data(), gao.size()));
    std::vector<double> bx(3 * (size_t)nbas);
    for (int i = 0; i < nbas; i++) {
        const double* r = env + atm[bas[i * BAS_SLOTS + ATOM_OF] * ATM_SLOTS + PTR_COORD];
        bx[i] = r[0];
        bx[nbas + i] = r[1];
        bx[2 * (size_t)nbas + i] = r[2];
    }
    CUDA_TRY(upload(&b->d_bas_x, bx.data(), bx.size()));

    // Schwarz matrix on the device
    CUDA_TRY(cudaMalloc(&b->d_qcond, sizeof(double) * (size_t)nbas * nbas));
    CUDA_TRY(cudaMemset(b->d_qcond, 0, sizeof(double) * (size_t)nbas * nbas));
    {
        std::vector<int> pi[JK_LMAX_ALL + 1][JK_LMAX_ALL + 1], pj[JK_LMAX_ALL + 1][JK_LMAX_ALL + 1];
        for (int i = 0; i < nbas; i++)
            for (int j = 0; j <= i; j++) {
                int li = bas[i * BAS_SLOTS + ANG_OF], lj = bas[j * BAS_SLOTS + ANG_OF];
                if (li >= lj) { pi[li][lj].push_back(i); pj[li][lj].push_back(j); }
                else { pi[lj][li].push_back(j); pj[lj][li].push_back(i); }
            }
        for (int a = 0; a <= JK_LMAX_ALL; a++)
            for (int c = 0; c <= a; c++) {
                int n = (int)pi[a][c].size();
                if (!n) continue;
                int *dpi, *dpj;
                CUDA_TRY(upload(&dpi, pi[a][c].data(), n));
                CUDA_TRY(upload(&dpj, pj[a][c].data(), n));
                if (a <= JK_LMAX)
                    g_qcond[a][c](dpi, dpj, n, b->d_atm, b->d_bas, b->d_env, nbas, b->d_qcond, b->rys, 0);
                else
                    jk_qcond_generic(dpi, dpj, n, b->d_atm, b->d_bas, b->d_env, nbas, b->d_qcond, b->rys, a, 0);
                cudaError_t e = cudaGetLastError();
                if (e == cudaSuccess) e = cudaDeviceSynchronize();
                cudaFree(dpi);
                cudaFree(dpj);
                CUDA_TRY(e);
            }
        b->h_qcond.resize((size_t)nbas * nbas);
        CUDA_TRY(cudaMemcpy(b->h_qcond.data(), b->d_qcond, sizeof(double) * (size_t)nbas * nbas,
                            cudaMemcpyDeviceToHost));
    }
    // Schwarz-sorted pair lists per lower-triangular group pair, in the
    // reference's class order (cuobc/scf/hf.py:343-389)
    const std::vector<double>& q = b->h_qcond;
    b->h_pair_locs.push_back(0);
    for (int gi = 0; gi < ngroups; gi++) {
        for (int gj = 0; gj <= gi; gj++) {
            std::vector<std::pair<double, long long>> lst;
            int p0 = group_off[gi], p1 = group_off[gi + 1], q0 = group_off[gj], q1 = group_off[gj + 1];
            for (int i = p0; i < p1; i++)
                for (int j = q0; j < q1; j++) {
                    if (gi == gj && !diag_block_with_triu && j > i) continue;
                    double v = q[(size_t)i * nbas + j];
                    if (v > cutoff) lst.push_back({v, (long long)i * nbas + j});
                }
            std::stable_sort(lst.begin(), lst.end(),
                             [](const std::pair<double, long long>& x, const std::pair<double, long long>& y) {
                                 return x.first > y.first;
                             });
            for (auto& e : lst) {
                b->h_pair2bra.push_back((int)(e.second / nbas));
                b->h_pair2ket.push_back((int)(e.second % nbas));
                double lq = log(e.first);
                b->h_log_q.push_back(lq > 0 ? 0 : lq);
                b->h_log_q_raw.push_back(lq);
            }
            b->h_cls_gi.push_back(gi);
            b->h_cls_gj.push_back(gj);
            b->h_pair_locs.push_back((int)b->h_pair2bra.size());
        }
    }
    b->ncp = (int)b->h_cls_gi.size();
    // primitive-pair data (cuobc/lib/gint/pair_data.c:83-141)
    long long npp = 0;
    b->h_prim_locs.push_back(0);
    for (int c = 0; c < b->ncp; c++) {
        int np12 = b->h_group_nprim[b->h_cls_gi[c]] * b->h_group_nprim[b->h_cls_gj[c]];
        npp += (long long)(b->h_pair_locs[c + 1] - b->h_pair_locs[c]) * np12;
        if (npp > 0x7fffffffLL) return set_err(JK_ERR_ARG, "too many primitive pairs");
        b->h_prim_locs.push_back((int)npp);
    }
    b->nprim_total = npp;
    std::vector<double> prim(6 * (size_t)(npp ? npp : 1));
    double *a12 = prim.data(), *e12 = a12 + npp, *x12 = e12 + npp, *y12 = x12 + npp, *z12 = y12 + npp;
    double* ia12 = z12 + npp;
    // single-precision copy for the FP32 quartets of the mixed mode; the
    // product centre is stored relative to the bra shell's centre so that
    // the small differences P - R_i keep their relative precision
    std::vector<float> primf(6 * (size_t)(npp ? npp : 1));
    b->h_pnp.assign(std::max<size_t>(b->h_pair2bra.size(), 1), 0);
    for (int c = 0; c < b->ncp; c++) {
        // primitive-major within the class: primitive k of pair r at
        // h_prim_locs[c] + k * (pairs in the class) + r
        const int p0 = b->h_pair_locs[c], pst = b->h_pair_locs[c + 1] - p0;
        for (int p = p0; p < p0 + pst; p++) {
            int ish = b->h_pair2bra[p], jsh = b->h_pair2ket[p];
            int npi = bas[ish * BAS_SLOTS + NPRIM_OF], npj = bas[jsh * BAS_SLOTS + NPRIM_OF];
            int li = bas[ish * BAS_SLOTS + ANG_OF], lj = bas[jsh * BAS_SLOTS + ANG_OF];
            const double* ai = env + bas[ish * BAS_SLOTS + PTR_EXP];
            const double* aj = env + bas[jsh * BAS_SLOTS + PTR_EXP];
            const double* ci = env + bas[ish * BAS_SLOTS + PTR_COEFF];
            const double* cj = env + bas[jsh * BAS_SLOTS + PTR_COEFF];
            const double* ri = env + atm[bas[ish * BAS_SLOTS + ATOM_OF] * ATM_SLOTS + PTR_COORD];
            const double* rj = env + atm[bas[jsh * BAS_SLOTS + ATOM_OF] * ATM_SLOTS + PTR_COORD];
            double norm = common_fac_sp(li) * common_fac_sp(lj);
            double dx = ri[0] - rj[0], dy = ri[1] - rj[1], dz = ri[2] - rj[2];
            double r2 = dx * dx + dy * dy + dz * dz;
            // primitive pairs whose Gaussian-product factor exp(-ai aj/(ai+aj) r^2)
            // is above exp(-JK_PRIM_EXPCUT) first, their count in h_pnp
            // (the thread kernels loop over those only; the others carry a
            // factor below 1e-26 and are kept after them for the kernels
            // that loop over all)
            std::vector<std::pair<int, int>> order;
            for (int pass = 0; pass < 2; pass++)
                for (int ip = 0; ip < npi; ip++)
                    for (int jp = 0; jp < npj; jp++) {
                        const bool kept = r2 * ai[ip] * aj[jp] / (ai[ip] + aj[jp]) <= JK_PRIM_EXPCUT;
                        if (kept == (pass == 0)) order.push_back({ip, jp});
                        if (pass == 0 && kept) b->h_pnp[p]++;
                    }
            long long off = b->h_prim_locs[c] + (p - p0);
            for (const auto& pr : order) {
                const int ip = pr.first, jp = pr.second;
                {
                    double aij = ai[ip] + aj[jp];
                    a12[off] = aij;
                    ia12[off] = 1. / aij;
                    e12[off] = norm * ci[ip] * cj[jp] * exp(-r2 * ai[ip] * aj[jp] / aij);
                    if (ish == jsh) e12[off] *= b->diag_fac;
                    x12[off] = (ai[ip] * ri[0] + aj[jp] * rj[0]) / aij;
                    y12[off] = (ai[ip] * ri[1] + aj[jp] * rj[1]) / aij;
                    z12[off] = (ai[ip] * ri[2] + aj[jp] * rj[2]) / aij;
                    primf[off] = (float)aij;
                    primf[npp + off] = (float)(1. / aij);
                    primf[2 * npp + off] = (float)(e12[off] / aij);
                    // P - R_i = aj (R_j - R_i) / (ai + aj)
                    primf[3 * npp + off] = (float)(aj[jp] * (rj[0] - ri[0]) / aij);
                    primf[4 * npp + off] = (float)(aj[jp] * (rj[1] - ri[1]) / aij);
                    primf[5 * npp + off] = (float)(aj[jp] * (rj[2] - ri[2]) / aij);
                }
                off += pst;
            }
        }
    }
    CUDA_TRY(upload(&b->d_pnp, b->h_pnp.data(), b->h_pnp.size()));
    CUDA_TRY(upload(&b->d_prim, prim.data(), prim.size()));
    CUDA_TRY(upload(&b->d_primf, primf.data(), primf.size()));
    {
        // pair geometry: the two shells' centres and first AOs per pair
        const size_t np = b->h_pair2bra.size();
        std::vector<double> geo(6 * (np ? np : 1));
        std::vector<int> pao(2 * (np ? np : 1));
        for (size_t p = 0; p < np; p++) {
            const int sh[2] = {b->h_pair2bra[p], b->h_pair2ket[p]};
            for (int a = 0; a < 2; a++) {
                for (int d = 0; d < 3; d++) geo[(3 * a + d) * np + p] = bx[(size_t)d * nbas + sh[a]];
                pao[a * np + p] = b->h_ao_loc[sh[a]];
            }
        }
        CUDA_TRY(upload(&b->d_pgeo, geo.data(), geo.size()));
        CUDA_TRY(upload(&b->d_pao, pao.data(), pao.size()));
    }
    CUDA_TRY(upload(&b->d_pair2bra, b->h_pair2bra.data(), b->h_pair2bra.size()));
    CUDA_TRY(upload(&b->d_pair2ket, b->h_pair2ket.data(), b->h_pair2ket.size()));
    CUDA_TRY(upload(&b->d_log_q, b->h_log_q.data(), b->h_log_q.size()));
    CUDA_TRY(upload(&b->d_log_q_raw, b->h_log_q_raw.data(), b->h_log_q_raw.size()));
    // class quartets (cp_ij >= cp_kl), each with its slice of the qoff buffer
    for (int cij = 0; cij < b->ncp; cij++)
        for (int ckl = 0; ckl <= cij; ckl++) {
            JKScreenCQ c;
            c.cp_ij = cij;
            c.cp_kl = ckl;
            c.gi = b->h_cls_gi[cij];
            c.gj = b->h_cls_gj[cij];
            c.gk = b->h_cls_gi[ckl];
            c.gl = b->h_cls_gj[ckl];
            c.pair_ij0 = b->h_pair_locs[cij];
            c.n_ij = b->h_pair_locs[cij + 1] - c.pair_ij0;
            c.pair_kl0 = b->h_pair_locs[ckl];
            c.n_kl = b->h_pair_locs[ckl + 1] - c.pair_kl0;
            if (c.n_ij == 0 || c.n_kl == 0) continue;
            c.qoff_off = b->qoff_total;
            b->qoff_total += c.n_ij + 1;
            b->h_cq.push_back(c);
            // unscreened work for shard plans: quartets x primitive
            // quartets x roots x Cartesian components (+ the digestion)
            const int l4[4] = {b->h_group_l[c.gi], b->h_group_l[c.gj], b->h_group_l[c.gk], b->h_group_l[c.gl]};
            double nf = 1.;
            for (int a = 0; a < 4; a++) nf *= (l4[a] + 1) * (l4[a] + 2) / 2;
            const double nq = cij == ckl ? 0.5 * c.n_ij * (c.n_ij + 1.) : (double)c.n_ij * c.n_kl;
            const double npq = (double)b->h_group_nprim[c.gi] * b->h_group_nprim[c.gj] * b->h_group_nprim[c.gk] *
                               b->h_group_nprim[c.gl];
            b->h_cq_cost.push_back(nq * (npq * ((l4[0] + l4[1] + l4[2] + l4[3]) / 2 + 1) * nf + 12. * nf));
        }
    b->ncq = (int)b->h_cq.size();
    CUDA_TRY(cudaMalloc(&b->d_qoff, sizeof(long long) * (b->qoff_total ? b->qoff_total : 1)));
    CUDA_TRY(cudaMalloc(&b->d_task0, sizeof(long long) * 2 * (b->ncq ? b->ncq : 1)));
    CUDA_TRY(cudaMalloc(&b->d_qoff32, sizeof(long long) * (b->qoff_total ? b->qoff_total : 1)));
    CUDA_TRY(cudaMalloc(&b->d_task032, sizeof(long long) * 2 * (b->ncq ? b->ncq : 1)));
    CUDA_TRY(cudaMalloc(&b->d_klb, sizeof(int) * (b->qoff_total ? b->qoff_total : 1)));
    CUDA_TRY(cudaMalloc(&b->d_dm_cond, sizeof(double) * ngroups * ngroups));
    for (int c = 0; c < b->ncq; c++) {
        JKScreenCQ& q = b->h_cq[c];
        q.ngroups = ngroups;
        q.lq_ij = b->d_log_q + q.pair_ij0;
        q.lq_kl = b->d_log_q + q.pair_kl0;
        q.rq_ij = b->d_log_q_raw + q.pair_ij0;
        q.rq_kl = b->d_log_q_raw + q.pair_kl0;
        q.dm_cond = b->d_dm_cond;
        q.qoff = b->d_qoff + q.qoff_off;
        q.qoff32 = b->d_qoff32 + q.qoff_off;
        q.klb = b->d_klb + q.qoff_off;
        q.task0 = b->d_task0 + 2 * c;
        q.task032 = b->d_task032 + 2 * c;
    }
    CUDA_TRY(upload(&b->d_cq, b->h_cq.data(), b->h_cq.size()));
    CUDA_TRY(cudaMalloc(&b->d_task01, sizeof(long long) * 2));
    // row prefixes of the per-class-pair entries: sized once for the largest
    // class, so those calls never free a buffer a queued kernel still reads
    {
        int mx = 1;
        for (int c = 0; c < b->ncp; c++) mx = std::max(mx, b->h_pair_locs[c + 1] - b->h_pair_locs[c]);
        CUDA_TRY(cudaMalloc(&b->d_qoff1, sizeof(long long) * (mx + 1)));
        b->qoff1_cap = mx + 1;
    }
    // pair-packed layout of the J side (jk_build)
    b->h_pack.clear();
    b->pack_total = 0;
    for (int c = 0; c < b->ncp; c++) {
        JKPackCls k;
        k.off = b->pack_total;
        k.pair0 = b->h_pair_locs[c];
        k.np = b->h_pair_locs[c + 1] - k.pair0;
        const int li = b->h_group_l[b->h_cls_gi[c]], lj = b->h_group_l[b->h_cls_gj[c]];
        k.nfi = (li + 1) * (li + 2) / 2;
        k.nfj = (lj + 1) * (lj + 2) / 2;
        b->pack_total += (long long)k.np * k.nfi * k.nfj;
        b->h_pack.push_back(k);
    }
    CUDA_TRY(upload(&b->d_pack, b->h_pack.data(), b->h_pack.size()));
    CUDA_TRY(b->fan.init());
    return JK_OK;
}

extern "C" int jk_basis_create(const int* atm, int natm, const int* bas, int nbas, const double* env, int nenv,
                               const int* group_offsets, int ngroups, double cutoff, int diag_block_with_triu,
                               jk_basis_t** out) {
    if (!atm || !bas || !env || !group_offsets || !out || natm <= 0 || nbas <= 0 || ngroups <= 0)
        return set_err(JK_ERR_ARG, "jk_basis_create: invalid arguments");
    jk_basis* b = new jk_basis();
    int rc = create_impl(atm, natm, bas, nbas, env, nenv, group_offsets, ngroups, cutoff, diag_block_with_triu, b);
    if (rc != JK_OK) {
        free_basis(b);
        *out = nullptr;
        return rc;
    }
    *out = b;
    return JK_OK;
}

extern "C" int jk_basis_destroy(jk_basis_t* b) {
    free_basis(b);
    return JK_OK;
}

extern "C" int jk_basis_info(const jk_basis_t* b, int* info) {
    if (!b || !info) return set_err(JK_ERR_ARG, "jk_basis_info: invalid arguments");
    info[0] = b->nbas;
    info[1] = b->nao;
    info[2] = b->ngroups;
    info[3] = b->ncp;
    info[4] = (int)b->h_pair2bra.size();
    info[5] = (int)b->nprim_total;
    info[6] = b->ncq;
    return JK_OK;
}

extern "C" int jk_basis_pairs(const jk_basis_t* b, int* pair2shls, int* pair_locs, double* log_q, double* q_cond) {
    if (!b) return set_err(JK_ERR_ARG, "jk_basis_pairs: null basis");
    size_t np = b->h_pair2bra.size();
    if (pair2shls) {
        std::copy(b->h_pair2bra.begin(), b->h_pair2bra.end(), pair2shls);
        std::copy(b->h_pair2ket.begin(), b->h_pair2ket.end(), pair2shls + np);
    }
    if (pair_locs) std::copy(b->h_pair_locs.begin(), b->h_pair_locs.end(), pair_locs);
    if (log_q) std::copy(b->h_log_q.begin(), b->h_log_q.end(), log_q);
    if (q_cond) std::copy(b->h_qcond.begin(), b->h_qcond.end(), q_cond);
    return JK_OK;
}

static void fill_seg(const jk_basis* b, int cp_ij, int cp_kl, const long long* qoff, int n_ij, const double* dm,
                     int n_dm, double* vj, double* vk, JKSeg* s) {
    s->rys = b->rys;
    s->qoff = qoff;
    s->kl_base = nullptr;
    s->n_ij = n_ij;
    s->pair_ij0 = b->h_pair_locs[cp_ij];
    s->pair_kl0 = b->h_pair_locs[cp_kl];
    s->prim_ij0 = b->h_prim_locs[cp_ij];
    s->prim_kl0 = b->h_prim_locs[cp_kl];
    s->nprim_ij = b->h_group_nprim[b->h_cls_gi[cp_ij]] * b->h_group_nprim[b->h_cls_gj[cp_ij]];
    s->nprim_kl = b->h_group_nprim[b->h_cls_gi[cp_kl]] * b->h_group_nprim[b->h_cls_gj[cp_kl]];
    s->pst_ij = b->h_pair_locs[cp_ij + 1] - b->h_pair_locs[cp_ij];
    s->pst_kl = b->h_pair_locs[cp_kl + 1] - b->h_pair_locs[cp_kl];
    s->nao = b->nao;
    s->n_dm = n_dm;
    s->pair2bra = b->d_pair2bra;
    s->pair2ket = b->d_pair2ket;
    long long n = b->nprim_total;
    s->a12 = b->d_prim;
    s->e12 = b->d_prim + n;
    s->x12 = b->d_prim + 2 * n;
    s->y12 = b->d_prim + 3 * n;
    s->z12 = b->d_prim + 4 * n;
    s->ia12 = b->d_prim + 5 * n;
    s->pf = b->d_primf;
    s->npf = n;
    s->bas_x = b->d_bas_x;
    s->pgeo = b->d_pgeo;
    s->pnp = b->d_pnp;
    s->pao = b->d_pao;
    s->npt = (int)b->h_pair2bra.size();
    s->nbas = b->nbas;
    s->ao_loc = b->d_ao_loc;
    s->dm = dm;
    s->vj = vj;
    s->vk = vk;
    s->dp_ij = s->dp_kl = nullptr;
    s->jp_ij = s->jp_kl = nullptr;
    s->np_ij = s->np_kl = 0;
    s->pk_stride = 0;
    s->ls[0] = b->h_group_l[b->h_cls_gi[cp_ij]];
    s->ls[1] = b->h_group_l[b->h_cls_gj[cp_ij]];
    s->ls[2] = b->h_group_l[b->h_cls_gi[cp_kl]];
    s->ls[3] = b->h_group_l[b->h_cls_gj[cp_kl]];
}

int jk_internal_class_index(const jk_basis_t* b, int cp_ij, int cp_kl);
static int class_index(const jk_basis* b, int cp_ij, int cp_kl) {
    int li = b->h_group_l[b->h_cls_gi[cp_ij]], lj = b->h_group_l[b->h_cls_gj[cp_ij]];
    int lk = b->h_group_l[b->h_cls_gi[cp_kl]], ll = b->h_group_l[b->h_cls_gj[cp_kl]];
    return JK_CLASS_INDEX(li, lj, lk, ll);
}

extern "C" int jk_shard_plan(const double* cost, int n, int nshards, int* owner) {
    if (n < 0 || nshards < 1 || (n > 0 && (!cost || !owner)))
        return set_err(JK_ERR_ARG, "jk_shard_plan: invalid arguments");
    std::vector<int> ord(n);
    for (int i = 0; i < n; i++) ord[i] = i;
    std::stable_sort(ord.begin(), ord.end(), [&](int a, int c) { return cost[a] > cost[c]; });
    std::vector<double> load(nshards, 0.);
    for (int i : ord) {
        int best = 0;
        for (int r = 1; r < nshards; r++)
            if (load[r] < load[best]) best = r;
        owner[i] = best;
        load[best] += cost[i];
    }
    return JK_OK;
}

// owner of every class quartet for nshards shards (cached per basis)
static const int* shard_owners(jk_basis* b, int nshards) {
    if (b->cq_owner_n != nshards || (int)b->h_cq_owner.size() != b->ncq) {
        b->h_cq_owner.assign(b->ncq, 0);
        jk_shard_plan(b->h_cq_cost.data(), b->ncq, nshards, b->h_cq_owner.data());
        b->cq_owner_n = nshards;
    }
    return b->h_cq_owner.data();
}

extern "C" int jk_build(jk_basis_t* b, const double* dm, int n_dm, double* vj, double* vk, const jk_opts_t* opts,
                        void* stream) {
    if (!b || !dm || n_dm <= 0) return set_err(JK_ERR_ARG, "jk_build: invalid arguments");
    if (!vj && !vk) return JK_OK;
    cudaStream_t st = (cudaStream_t)stream;
    double tol = opts ? opts->direct_scf_tol : b->cutoff;
    int nbins = opts && opts->nbins > 0 ? opts->nbins : 10;
    int prescreen = opts ? opts->prescreen : 1;
    dim3 gg(b->ngroups, b->ngroups);
    jk_dm_cond_kernel<<<gg, 256, 0, st>>>(dm, b->nao, n_dm, b->d_group_ao, b->ngroups, b->d_dm_cond);
    CUDA_TRY(cudaGetLastError());
    if (b->ncq == 0) return JK_OK;
    double fp32_cutoff = opts ? opts->fp32_cutoff : 0.;
    jk_screen_kernel<<<b->ncq, 256, 0, st>>>(b->d_cq, tol, nbins, prescreen, fp32_cutoff);
    CUDA_TRY(cudaGetLastError());
    // pair-packed density and J accumulators for the thread kernels
    const bool packed = vj && b->pack_total > 0;
    double *dp = nullptr, *jp = nullptr;
    const int pk_blocks = (int)std::min<long long>((b->pack_total + 255) / 256, (long long)b->nsm * 8);
    if (packed) {
        const size_t need = (size_t)2 * n_dm * b->pack_total;
        if (need > b->pk_cap) {
            cudaFree(b->d_pk);
            b->d_pk = nullptr;
            CUDA_TRY(cudaMalloc(&b->d_pk, sizeof(double) * need));
            b->pk_cap = need;
        }
        dp = b->d_pk;
        jp = b->d_pk + (size_t)n_dm * b->pack_total;
        jk_pack_kernel<<<pk_blocks, 256, 0, st>>>(b->d_pack, b->ncp, b->pack_total, b->d_pair2bra, b->d_pair2ket,
                                                   b->d_ao_loc, dm, b->nao, n_dm, dp, nullptr, nullptr, 0);
        CUDA_TRY(cudaGetLastError());
        CUDA_TRY(cudaMemsetAsync(jp, 0, sizeof(double) * n_dm * b->pack_total, st));
    }
    const int nshards = opts && opts->nshards > 1 ? opts->nshards : 1;
    const int shard = opts ? opts->shard : 0;
    if (nshards > 1 && (shard < 0 || shard >= nshards)) return set_err(JK_ERR_ARG, "jk_build: shard out of range");
    const int* owner = nshards > 1 ? shard_owners(b, nshards) : nullptr;
    CUDA_TRY(b->fan.begin(st));
    for (int c = 0; c < b->ncq; c++) {
        if (owner && owner[c] != shard) continue;
        const JKScreenCQ& cq = b->h_cq[c];
        JKSeg seg;
        fill_seg(b, cq.cp_ij, cq.cp_kl, b->d_qoff + cq.qoff_off, cq.n_ij, dm, n_dm, vj, vk, &seg);
        if (packed) {
            const JKPackCls &ki = b->h_pack[cq.cp_ij], &kk = b->h_pack[cq.cp_kl];
            seg.dp_ij = dp + ki.off;
            seg.dp_kl = dp + kk.off;
            seg.jp_ij = jp + ki.off;
            seg.jp_kl = jp + kk.off;
            seg.np_ij = ki.np;
            seg.np_kl = kk.np;
            seg.pk_stride = b->pack_total;
        }
        long long maxt = cq.cp_ij == cq.cp_kl ? (long long)cq.n_ij * (cq.n_ij + 1) / 2
                                              : (long long)cq.n_ij * cq.n_kl;
        int ci = class_index(b, cq.cp_ij, cq.cp_kl);
        jk_launch_fn fn = g_tab64[ci];
        if (!fn) return set_err(JK_ERR_UNSUPPORTED, "no kernel for class quartet %d", c);
        CUDA_TRY(fn(seg, b->d_task0 + 2 * c, maxt, b->nsm, b->fan.pick(2 * c)));
        if (fp32_cutoff > 0) {
            jk_launch_fn f32 = g_tab32[ci];
            if (!f32) return set_err(JK_ERR_UNSUPPORTED, "no FP32 kernel for class quartet %d", c);
            seg.qoff = b->d_qoff32 + cq.qoff_off;
            seg.kl_base = b->d_klb + cq.qoff_off;
            CUDA_TRY(f32(seg, b->d_task032 + 2 * c, maxt, b->nsm, b->fan.pick(2 * c + 1)));
        }
    }
    CUDA_TRY(b->fan.end(st));
    if (packed) {
        jk_pack_kernel<<<pk_blocks, 256, 0, st>>>(b->d_pack, b->ncp, b->pack_total, b->d_pair2bra, b->d_pair2ket,
                                                   b->d_ao_loc, dm, b->nao, n_dm, nullptr, jp, vj, 1);
        CUDA_TRY(cudaGetLastError());
    }
    return JK_OK;
}

// Row prefix of one class pair's task list from the host bins of the
// per-class-pair entries (nr_jk_driver.cu:252-280, nr_fill_ao_ints.cu:519-545):
// row ij in bin s (ij[s] <= ij < ij[s+1]) keeps c_s = kl[nbins - s] - kl[0]
// columns (none when kl[0] != 0: the reference's bins start at 0), at most
// ij + 1 of them on a diagonal class pair of jk_build_class_pair; rows below
// ij[0] or from ij[nbins] on keep none.  The bins go to the device by value,
// so the entries neither copy nor synchronise.
#define JK_ROWBINS_MAX 64
struct JKRowBins {
    int nbins, diag;
    int ij[JK_ROWBINS_MAX + 1], kl[JK_ROWBINS_MAX + 1];
};

// tasks of rows [0, r)
__host__ __device__ inline long long jk_rowbins_tasks(const JKRowBins& b, long long r) {
    if (b.kl[0] != 0) return 0;
    long long acc = 0;
    for (int s = 0; s < b.nbins; s++) {
        const long long lo = b.ij[s];
        const long long hi = r < b.ij[s + 1] ? r : b.ij[s + 1];
        if (hi <= lo) continue;
        const long long c = b.kl[b.nbins - s] - b.kl[0];
        if (!b.diag) {
            acc += c * (hi - lo);
        } else {
            // rows below c keep row + 1 columns, the others c
            const long long m = lo > (c < hi ? c : hi) ? lo : (c < hi ? c : hi);
            acc += (m * (m + 1) - lo * (lo + 1)) / 2 + c * (hi - m);
        }
    }
    return acc;
}

__global__ void jk_rowbins_kernel(const JKRowBins rb, int n_ij, long long* __restrict__ qoff,
                                  long long* __restrict__ task0) {
    for (long long r = blockIdx.x * (long long)blockDim.x + threadIdx.x; r <= n_ij;
         r += (long long)gridDim.x * blockDim.x)
        qoff[r] = jk_rowbins_tasks(rb, r);
    if (blockIdx.x == 0 && threadIdx.x == 0) {
        task0[0] = 0;
        task0[1] = jk_rowbins_tasks(rb, n_ij);
    }
}

// bins of a per-class-pair call -> the basis's row prefix and task count, on
// `st`; returns the task count through *tot
static int class_pair_rows(jk_basis* b, const int* bins_ij, const int* bins_kl, int nbins, int n_ij, int diag,
                           cudaStream_t st, long long* tot) {
    if (nbins > JK_ROWBINS_MAX) return set_err(JK_ERR_ARG, "nbins %d above %d", nbins, JK_ROWBINS_MAX);
    JKRowBins rb;
    rb.nbins = nbins;
    rb.diag = diag;
    for (int s = 0; s <= nbins; s++) {
        rb.ij[s] = bins_ij[s];
        rb.kl[s] = bins_kl[s];
        if (s && (bins_ij[s] < bins_ij[s - 1] || bins_kl[s] < bins_kl[s - 1]))
            return set_err(JK_ERR_ARG, "bins must not decrease");
    }
    if (n_ij + 1 > (int)b->qoff1_cap) return set_err(JK_ERR_ARG, "class pair larger than the basis' classes");
    *tot = jk_rowbins_tasks(rb, n_ij);
    const int blocks = (int)std::min<long long>((n_ij + 256) / 256, (long long)b->nsm * 4);
    jk_rowbins_kernel<<<blocks, 256, 0, st>>>(rb, n_ij, b->d_qoff1, b->d_task01);
    CUDA_TRY(cudaGetLastError());
    return JK_OK;
}

extern "C" int jk_class_pair_tasks(const int* bins_ij, const int* bins_kl, int nbins, int n_ij, int diag,
                                   long long* qoff, long long* total) {
    if (!bins_ij || !bins_kl || nbins <= 0 || nbins > JK_ROWBINS_MAX || n_ij < 0 || !total)
        return set_err(JK_ERR_ARG, "jk_class_pair_tasks: invalid arguments");
    JKRowBins rb;
    rb.nbins = nbins;
    rb.diag = diag ? 1 : 0;
    for (int s = 0; s <= nbins; s++) {
        rb.ij[s] = bins_ij[s];
        rb.kl[s] = bins_kl[s];
        if (s && (bins_ij[s] < bins_ij[s - 1] || bins_kl[s] < bins_kl[s - 1]))
            return set_err(JK_ERR_ARG, "bins must not decrease");
    }
    if (qoff)
        for (int r = 0; r <= n_ij; r++) qoff[r] = jk_rowbins_tasks(rb, r);
    *total = jk_rowbins_tasks(rb, n_ij);
    return JK_OK;
}

extern "C" int jk_build_class_pair(jk_basis_t* b, double* vj, double* vk, const double* dm, int nao, int n_dm,
                                   const int* bins_locs_ij, const int* bins_locs_kl, int nbins, int cp_ij,
                                   int cp_kl, void* stream) {
    if (!b || !dm || !bins_locs_ij || !bins_locs_kl || nbins <= 0) return set_err(JK_ERR_ARG, "invalid arguments");
    if (nao != b->nao) return set_err(JK_ERR_ARG, "nao %d does not match the basis (%d)", nao, b->nao);
    if (cp_ij < 0 || cp_ij >= b->ncp || cp_kl < 0 || cp_kl > cp_ij) return set_err(JK_ERR_ARG, "bad class pair");
    if (!vj && !vk) return JK_OK;
    cudaStream_t st = (cudaStream_t)stream;
    int n_ij = b->h_pair_locs[cp_ij + 1] - b->h_pair_locs[cp_ij];
    // kl bin kb pairs with ij in [bins_ij[0], bins_ij[nbins - kb]) (nr_jk_driver.cu:252-280):
    // row ij (in bin sij) keeps kl < bins_kl[nbins - sij]; diagonal classes keep kl <= ij
    jk_launch_fn fn = g_tab64[class_index(b, cp_ij, cp_kl)];
    if (!fn) return set_err(JK_ERR_UNSUPPORTED, "no kernel for this class pair");
    long long tot = 0;
    int rc = class_pair_rows(b, bins_locs_ij, bins_locs_kl, nbins, n_ij, cp_ij == cp_kl, st, &tot);
    if (rc) return rc;
    JKSeg seg;
    fill_seg(b, cp_ij, cp_kl, b->d_qoff1, n_ij, dm, n_dm, vj, vk, &seg);
    CUDA_TRY(fn(seg, b->d_task01, tot, b->nsm, st));
    return JK_OK;
}

// ERI tensor of one class pair (jk_generic.cu)
cudaError_t jk_launch_fill(const JKSeg& seg, const long long* task0, long long max_tasks, int nsm, double* eri,
                           const long long* strides, const int* offsets, cudaStream_t st);

extern "C" int jk_fill_int2e(jk_basis_t* b, double* eri, int nao, const int* strides, const int* ao_offsets,
                             const int* bins_locs_ij, const int* bins_locs_kl, int nbins, int cp_ij, int cp_kl,
                             void* stream) {
    if (!b || !eri || !strides || !ao_offsets || !bins_locs_ij || !bins_locs_kl || nbins <= 0)
        return set_err(JK_ERR_ARG, "jk_fill_int2e: invalid arguments");
    if (nao != b->nao) return set_err(JK_ERR_ARG, "nao %d does not match the basis (%d)", nao, b->nao);
    // any two class pairs (the two-centre metric of int3c.get_int2c pairs
    // auxiliary classes in both orders)
    if (cp_ij < 0 || cp_ij >= b->ncp || cp_kl < 0 || cp_kl >= b->ncp) return set_err(JK_ERR_ARG, "bad class pair");
    cudaStream_t st = (cudaStream_t)stream;
    const int n_ij = b->h_pair_locs[cp_ij + 1] - b->h_pair_locs[cp_ij];
    // kl bin kb pairs with ij in [bins_ij[0], bins_ij[nbins - kb]): row ij (in
    // bin sij) keeps kl < bins_kl[nbins - sij] (nr_fill_ao_ints.cu:519-545)
    long long tot = 0;
    int rc = class_pair_rows(b, bins_locs_ij, bins_locs_kl, nbins, n_ij, 0, st, &tot);
    if (rc) return rc;
    JKSeg seg;
    fill_seg(b, cp_ij, cp_kl, b->d_qoff1, n_ij, nullptr, 0, nullptr, nullptr, &seg);
    long long s64[4];
    for (int a = 0; a < 4; a++) s64[a] = strides[a];
    CUDA_TRY(jk_launch_fill(seg, b->d_task01, tot, b->nsm, eri, s64, ao_offsets, st));
    return JK_OK;
}

// row-major C[M,N] = alpha op(A) op(B) + beta C through column-major cuBLAS
static cublasStatus_t gemm_rm(cublasHandle_t h, bool ta, bool tb, int M, int N, int K, double alpha,
                              const double* A, int lda, const double* B, int ldb, double beta, double* C, int ldc) {
    return cublasDgemm(h, tb ? CUBLAS_OP_T : CUBLAS_OP_N, ta ? CUBLAS_OP_T : CUBLAS_OP_N, N, M, K, &alpha, B, ldb,
                       A, lda, &beta, C, ldc);
}

#define BLAS_TRY(x)                                                              \
    do {                                                                         \
        cublasStatus_t s_ = (x);                                                 \
        if (s_ != CUBLAS_STATUS_SUCCESS) return set_err(JK_ERR_CUDA, "%s: cublas status %d", #x, (int)s_); \
    } while (0)

extern "C" int jk_get_jk(jk_basis_t* b, const double* coeff, int nao0, const double* dm0, int n_dm, double* vj0,
                         double* vk0, const jk_opts_t* opts, void* stream) {
    if (!b || !coeff || !dm0 || n_dm <= 0 || nao0 <= 0) return set_err(JK_ERR_ARG, "jk_get_jk: invalid arguments");
    cudaStream_t st = (cudaStream_t)stream;
    int nao = b->nao;
    size_t nn = (size_t)nao * nao * n_dm;
    size_t need = 4 * nn + (size_t)nao * nao0;
    if (need > b->work_cap) {
        cudaFree(b->d_work);
        b->d_work = nullptr;
        CUDA_TRY(cudaMalloc(&b->d_work, sizeof(double) * need));
        b->work_cap = need;
    }
    if (!b->blas) BLAS_TRY(cublasCreate(&b->blas));
    BLAS_TRY(cublasSetStream(b->blas, st));
    double* dms = b->d_work;
    double* vjw = dms + nn;
    double* vkw = vjw + nn;
    double* sym = vkw + nn;
    double* tmp = sym + nn;  // nao x nao0
    // dms = C D C^T (cuobc/scf/hf.py:73-74)
    for (int m = 0; m < n_dm; m++) {
        const double* D = dm0 + (size_t)m * nao0 * nao0;
        BLAS_TRY(gemm_rm(b->blas, false, false, nao, nao0, nao0, 1.0, coeff, nao0, D, nao0, 0.0, tmp, nao0));
        BLAS_TRY(gemm_rm(b->blas, false, true, nao, nao, nao0, 1.0, tmp, nao0, coeff, nao0, 0.0,
                         dms + (size_t)m * nao * nao, nao));
    }
    if (vj0) CUDA_TRY(cudaMemsetAsync(vjw, 0, sizeof(double) * nn, st));
    if (vk0) CUDA_TRY(cudaMemsetAsync(vkw, 0, sizeof(double) * nn, st));
    int rc = jk_build(b, dms, n_dm, vj0 ? vjw : nullptr, vk0 ? vkw : nullptr, opts, stream);
    if (rc) return rc;
    // J = 2 C^T (V + V^T) C, K = C^T (V + V^T) C (cuobc/scf/hf.py:171-181)
    for (int pass = 0; pass < 2; pass++) {
        double* out = pass == 0 ? vj0 : vk0;
        double* w = pass == 0 ? vjw : vkw;
        if (!out) continue;
        jk_symmetrize_kernel<<<b->nsm * 4, 256, 0, st>>>(w, sym, nao, n_dm, pass == 0 ? 2.0 : 1.0);
        CUDA_TRY(cudaGetLastError());
        for (int m = 0; m < n_dm; m++) {
            BLAS_TRY(gemm_rm(b->blas, false, false, nao, nao0, nao, 1.0, sym + (size_t)m * nao * nao, nao, coeff,
                             nao0, 0.0, tmp, nao0));
            BLAS_TRY(gemm_rm(b->blas, true, false, nao0, nao0, nao, 1.0, coeff, nao0, tmp, nao0, 0.0,
                             out + (size_t)m * nao0 * nao0, nao0));
        }
    }
    return JK_OK;
}

// ---------------------------------------------------------------------------
// introspection for the bench and the tests
// ---------------------------------------------------------------------------
// per class quartet: cp_ij, cp_kl, li, lj, lk, ll, nprim_ij, nprim_kl
extern "C" int jk_basis_cq_info(const jk_basis_t* b, int* out) {
    if (!b || !out) return set_err(JK_ERR_ARG, "jk_basis_cq_info: invalid arguments");
    for (int c = 0; c < b->ncq; c++) {
        const JKScreenCQ& cq = b->h_cq[c];
        int* o = out + 8 * c;
        o[0] = cq.cp_ij;
        o[1] = cq.cp_kl;
        o[2] = b->h_group_l[cq.gi];
        o[3] = b->h_group_l[cq.gj];
        o[4] = b->h_group_l[cq.gk];
        o[5] = b->h_group_l[cq.gl];
        o[6] = b->h_group_nprim[cq.gi] * b->h_group_nprim[cq.gj];
        o[7] = b->h_group_nprim[cq.gk] * b->h_group_nprim[cq.gl];
    }
    return JK_OK;
}

// screened contracted-quartet counts of the last jk_build, per class quartet
extern "C" int jk_last_counts(const jk_basis_t* b, long long* out, void* stream) {
    if (!b || !out) return set_err(JK_ERR_ARG, "jk_last_counts: invalid arguments");
    if (b->ncq == 0) return JK_OK;
    std::vector<long long> t(2 * (size_t)b->ncq), t32(2 * (size_t)b->ncq);
    CUDA_TRY(cudaMemcpyAsync(t.data(), b->d_task0, sizeof(long long) * t.size(), cudaMemcpyDeviceToHost,
                             (cudaStream_t)stream));
    CUDA_TRY(cudaMemcpyAsync(t32.data(), b->d_task032, sizeof(long long) * t32.size(), cudaMemcpyDeviceToHost,
                             (cudaStream_t)stream));
    CUDA_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    // FP64 quartets in out[0..ncq), FP32 quartets (mixed mode) in out[ncq..2 ncq)
    for (int c = 0; c < b->ncq; c++) {
        out[c] = t[2 * c + 1];
        out[b->ncq + c] = t32[2 * c + 1];
    }
    return JK_OK;
}

// FMA-pipe peak: 8 independent FMA chains per thread, whole device
template <typename T>
__global__ void jk_fma_peak_kernel(T* out, int iters) {
    T a[8];
#pragma unroll
    for (int k = 0; k < 8; k++) a[k] = (T)(threadIdx.x * 1e-7 + k);
    const T b = (T)0.9999999, c = (T)1e-7;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
#pragma unroll
            for (int k = 0; k < 8; k++) a[k] = fma(a[k], b, c);
        }
    }
    T s = 0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += a[k];
    if (s == (T)-1) out[0] = s;  // keeps the chains alive
}

extern "C" int jk_fma_peak(int fp32, double* tflops) {
    if (!tflops) return set_err(JK_ERR_ARG, "jk_fma_peak: null output");
    int dev, nsm;
    CUDA_TRY(cudaGetDevice(&dev));
    CUDA_TRY(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
    void* buf;
    CUDA_TRY(cudaMalloc(&buf, 16));
    cudaEvent_t e0, e1;
    CUDA_TRY(cudaEventCreate(&e0));
    CUDA_TRY(cudaEventCreate(&e1));
    const int iters = 4096, threads = 256, blocks = nsm * 8;
    double best = 0;
    for (int rep = 0; rep < 4; rep++) {
        CUDA_TRY(cudaEventRecord(e0));
        if (fp32) jk_fma_peak_kernel<float><<<blocks, threads>>>((float*)buf, iters);
        else jk_fma_peak_kernel<double><<<blocks, threads>>>((double*)buf, iters);
        CUDA_TRY(cudaEventRecord(e1));
        CUDA_TRY(cudaEventSynchronize(e1));
        float ms;
        CUDA_TRY(cudaEventElapsedTime(&ms, e0, e1));
        double flops = 2.0 * 8 * 16 * (double)iters * threads * blocks;
        if (rep > 0 && flops / (ms * 1e-3) / 1e12 > best) best = flops / (ms * 1e-3) / 1e12;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(buf);
    *tflops = best;
    return JK_OK;
}

// device evaluation of the Rys tables at a batch of points, through the
// paths the kernels use: mode 0 all roots from the shared-memory copy (thread
// kernels), 1 one root at a time from it (team kernels), 2 one root from the
// global table (setup kernels), 3 all roots in single precision (the FP32
// quartets of the mixed mode, n <= JK_F32_ROOTS; thread kernels), 4 one root
// at a time in single precision (team kernels)
template <int N>
__global__ void jk_rys_eval_kernel(const double* rys, const double* x, int count, double* s, double* w, int mode) {
    extern __shared__ __align__(16) double tab[];
    if (mode >= 3) rys_table_to_smem_f<N>(rys, reinterpret_cast<float*>(tab));
    else rys_table_to_smem<N>(rys, tab);
    __syncthreads();
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    if (mode == 3) {
        if constexpr (N <= JK_F32_ROOTS) {
            float rs[N], rw[N];
            rys_roots_all_f<N>(reinterpret_cast<const float*>(tab), (float)x[i], rs, rw);
            for (int r = 0; r < N; r++) {
                s[i * N + r] = rs[r];
                w[i * N + r] = rw[r];
            }
        }
    } else if (mode == 4) {
        if constexpr (N <= JK_F32_ROOTS) {
            for (int r = 0; r < N; r++) {
                float rs, rw;
                rys_root_one_f<N>(reinterpret_cast<const float*>(tab), (float)x[i], r, rs, rw);
                s[i * N + r] = rs;
                w[i * N + r] = rw;
            }
        }
    } else if (mode == 5) {  // run-time root count (generic kernels), global table
        for (int r = 0; r < N; r++) {
            double rs, rw;
            rys_root_rt(rys, N, x[i], r, rs, rw);
            s[i * N + r] = rs;
            w[i * N + r] = rw;
        }
    } else if (mode == 0) {
        double rs[N], rw[N];
        rys_roots_all<N>(tab, x[i], rs, rw);
        for (int r = 0; r < N; r++) {
            s[i * N + r] = rs[r];
            w[i * N + r] = rw[r];
        }
    } else {
        for (int r = 0; r < N; r++) {
            if (mode == 1) rys_root_one<N>(tab, x[i], r, s[i * N + r], w[i * N + r]);
            else rys_root<N>(rys, x[i], r, s[i * N + r], w[i * N + r]);
        }
    }
}

template <int N>
static cudaError_t rys_eval_launch(const double* rys, const double* x, int count, double* s, double* w, int mode,
                                   cudaStream_t st) {
    size_t smem = RysS<N>::WORDS * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(jk_rys_eval_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    jk_rys_eval_kernel<N><<<(count + 127) / 128, 128, smem, st>>>(rys, x, count, s, w, mode);
    return cudaGetLastError();
}

extern "C" int jk_rys_roots_device(int n, const double* x, int count, double* s, double* w, int mode, void* stream) {
    if (n < 1 || n > RYS_NMAX || !x || !s || !w || count < 0 || mode < 0 || mode > 5 ||
        ((mode == 3 || mode == 4) && n > JK_F32_ROOTS))
        return set_err(JK_ERR_ARG, "jk_rys_roots_device: bad args");
    if (count == 0) return JK_OK;
    const double* rys;
    int rc = rys_table_device(&rys);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    cudaError_t e;
    switch (n) {
        case 1: e = rys_eval_launch<1>(rys, x, count, s, w, mode, st); break;
        case 2: e = rys_eval_launch<2>(rys, x, count, s, w, mode, st); break;
        case 3: e = rys_eval_launch<3>(rys, x, count, s, w, mode, st); break;
        case 4: e = rys_eval_launch<4>(rys, x, count, s, w, mode, st); break;
        case 5: e = rys_eval_launch<5>(rys, x, count, s, w, mode, st); break;
        case 6: e = rys_eval_launch<6>(rys, x, count, s, w, mode, st); break;
        case 7: e = rys_eval_launch<7>(rys, x, count, s, w, mode, st); break;
        case 8: e = rys_eval_launch<8>(rys, x, count, s, w, mode, st); break;
        case 9: e = rys_eval_launch<9>(rys, x, count, s, w, mode, st); break;
        case 10: e = rys_eval_launch<10>(rys, x, count, s, w, mode, st); break;
        case 11: e = rys_eval_launch<11>(rys, x, count, s, w, mode, st); break;
        case 12: e = rys_eval_launch<12>(rys, x, count, s, w, mode, st); break;
        default: e = rys_eval_launch<13>(rys, x, count, s, w, mode, st); break;
    }
    CUDA_TRY(e);
    return JK_OK;
}

// ---------------------------------------------------------------------------
// internal helpers for the other translation units
// ---------------------------------------------------------------------------
int jk_internal_set_err(int code, const char* msg) { return set_err(code, "%s", msg); }

int jk_internal_class_info(const jk_basis_t* b, int cp_ij, int cp_kl, int* n_ij, int* n_kl, int* nao) {
    if (!b || cp_ij < 0 || cp_ij >= b->ncp || cp_kl < 0 || cp_kl > cp_ij)
        return set_err(JK_ERR_ARG, "bad class pair (%d, %d)", cp_ij, cp_kl);
    *n_ij = b->h_pair_locs[cp_ij + 1] - b->h_pair_locs[cp_ij];
    *n_kl = b->h_pair_locs[cp_kl + 1] - b->h_pair_locs[cp_kl];
    *nao = b->nao;
    return JK_OK;
}

void jk_internal_fill_seg(const jk_basis_t* b, int cp_ij, int cp_kl, const long long* qoff, int n_ij,
                          const double* dm, int n_dm, double* vj, double* vk, JKSeg* out) {
    fill_seg(b, cp_ij, cp_kl, qoff, n_ij, dm, n_dm, vj, vk, out);
}

int jk_internal_launch(const jk_basis_t* b, int cp_ij, int cp_kl, const JKSeg& seg, const long long* d_task0,
                       long long max_tasks, void* stream) {
    jk_launch_fn fn = g_tab64[class_index(b, cp_ij, cp_kl)];
    if (!fn) return set_err(JK_ERR_UNSUPPORTED, "no kernel for class pair (%d, %d)", cp_ij, cp_kl);
    CUDA_TRY(fn(seg, d_task0, max_tasks, b->nsm, (cudaStream_t)stream));
    return JK_OK;
}

int jk_internal_launch_part(int class_idx, int fp32, const JKSeg& seg, const long long* d_task0, long long max_tasks,
                            int nsm, void* stream) {
    init_tables();
    jk_launch_fn fn = fp32 ? g_tab32[class_idx] : g_tab64[class_idx];
    if (!fn) return set_err(JK_ERR_UNSUPPORTED, "no kernel for class %d", class_idx);
    CUDA_TRY(fn(seg, d_task0, max_tasks, nsm, (cudaStream_t)stream));
    return JK_OK;
}

int jk_internal_class_index(const jk_basis_t* b, int cp_ij, int cp_kl) { return class_index(b, cp_ij, cp_kl); }

jk_launch_batch_fn jk_internal_batch_launcher(int class_idx, int fp32) {
    init_tables();
    return fp32 ? g_tabs.b32[class_idx] : g_tabs.b64[class_idx];
}

int jk_internal_class_team(int class_idx) {
    init_tables();
    return g_tabs.team[class_idx];
}

jk_fill_fn jk_internal_fill_launcher(int class_idx) {
    init_tables();
    return g_tabs.fill[class_idx];
}

void jk_internal_fill_seg_batch(const jk_basis_t* b, int c, const double* dm, int n_dm, double* vj, double* vk,
                                int fp32, JKSeg* out) {
    const JKScreenCQ& cq = b->h_cq[c];
    fill_seg(b, cq.cp_ij, cq.cp_kl, fp32 ? cq.qoff32 : cq.qoff, cq.n_ij, dm, n_dm, vj, vk, out);
    if (fp32) out->kl_base = cq.klb;
}

int jk_internal_pack_batch(const JKPackMol* d_mols, int nmol, long long max_total, int mode, void* stream) {
    if (nmol <= 0 || max_total <= 0) return JK_OK;
    const unsigned bx = (unsigned)std::min<long long>((max_total + 255) / 256, 64);
    jk_pack_batch_kernel<<<dim3(bx, nmol), 256, 0, (cudaStream_t)stream>>>(d_mols, mode);
    CUDA_TRY(cudaGetLastError());
    return JK_OK;
}

int jk_internal_screen(const JKScreenCQ* d_cq, int ncq, double tol, int nbins, int prescreen, double fp32_cutoff,
                       void* stream) {
    if (ncq <= 0) return JK_OK;
    jk_screen_kernel<<<ncq, 256, 0, (cudaStream_t)stream>>>(d_cq, tol, nbins, prescreen, fp32_cutoff);
    CUDA_TRY(cudaGetLastError());
    return JK_OK;
}
