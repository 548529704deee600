// Batched J/K builds: many molecules (one jk_basis each) in one pass.
//
// The single-molecule path launches one kernel per class quartet; for small
// molecules those launches are tiny and the GPU idles between them.  Here the
// class quartets of all molecules that share a class key (the four angular
// momenta and the two primitive counts) become segments of ONE launch, so a
// batch of hundreds of molecules costs one launch per class key plus three
// bookkeeping launches (density condensation, screening, segment prefixes),
// all on one stream with no host synchronisation; the whole sequence can be
// captured into a CUDA graph and replayed every SCF iteration.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <map>
#include <tuple>
#include <vector>

#include "jk_internal.h"

#define BCUDA(x)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (x);                                                                      \
        if (e_ != cudaSuccess) return jk_internal_set_err(JK_ERR_CUDA, cudaGetErrorString(e_));    \
    } while (0)

struct JKDmCond {
    const double* dm;
    const int* gao;  // group AO offsets (device)
    double* out;     // ngroups x ngroups
    int nao, n_dm, ngroups;
};

struct JKSym {
    const double* in;
    double* out;
    int nao, n_dm;
};

struct JKBatchKey {
    int cls, np_ij, np_kl;
    std::vector<std::pair<int, int>> segs;  // (molecule, class quartet)
    long long max_tasks = 0;
};

struct jk_batch {
    int device = 0, nsm = 148, nmol = 0, max_groups = 0;
    std::vector<jk_basis*> mols;
    std::vector<JKBatchKey> keys;
    std::vector<int> key_off;  // nkeys + 1 segment offsets
    int nseg = 0;
    JKScreenCQ* d_cq = nullptr;
    int ncq = 0;
    JKDmCond* d_dmc = nullptr;
    std::vector<JKDmCond> h_dmc;
    JKSeg *d_seg64 = nullptr, *d_seg32 = nullptr;
    long long *d_segt64 = nullptr, *d_segt32 = nullptr;
    const long long **d_cnt64 = nullptr, **d_cnt32 = nullptr;
    int* d_key_off = nullptr;
    // pointer set the segment tables were built for
    std::vector<const double*> seg_dm;
    std::vector<double*> seg_vj, seg_vk;
    int seg_ndm = -1;
    // transform workspace
    cublasHandle_t blas = nullptr;
    double* d_work = nullptr;
    size_t work_cap = 0;
    JKSym* d_sym = nullptr;
    std::vector<size_t> w_dms, w_vj, w_vk, w_sym, w_tmp;  // offsets per molecule
    int w_ndm = -1;
    // captured graph
    cudaGraphExec_t graph = nullptr;
    JKFanout fan;  // side streams of the class launches
    // pair-packed J side: every molecule's packed densities, then every
    // molecule's packed J accumulators (one memset clears them all)
    double* d_pk = nullptr;
    size_t pk_cap = 0, pk_jp = 0;  // capacity; first accumulator element
    JKPackMol* d_pmol = nullptr;
    long long pk_max = 0;          // largest per-molecule packed size
    bool packed = false;
};

// per (molecule, gi, gj): max |D| over the group block (blockIdx.z = molecule)
__global__ void jk_dm_cond_batch_kernel(const JKDmCond* __restrict__ t) {
    const JKDmCond m = t[blockIdx.z];
    int gi = blockIdx.x, gj = blockIdx.y;
    if (gi >= m.ngroups || gj >= m.ngroups) return;
    int p0 = m.gao[gi], p1 = m.gao[gi + 1], q0 = m.gao[gj], q1 = m.gao[gj + 1];
    int np = p1 - p0, nq = q1 - q0;
    double mx = 0;
    long long n = (long long)np * nq * m.n_dm;
    for (long long e = threadIdx.x; e < n; e += blockDim.x) {
        int idm = (int)(e / ((long long)np * nq));
        int rem = (int)(e - (long long)idm * np * nq);
        int p = p0 + rem / nq, q = q0 + rem % nq;
        mx = fmax(mx, fabs(m.dm[(size_t)idm * m.nao * m.nao + (size_t)p * m.nao + q]));
    }
    __shared__ double red[256];
    red[threadIdx.x] = mx;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] = fmax(red[threadIdx.x], red[threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) m.out[gi * m.ngroups + gj] = red[0];
}

// exclusive prefix of the per-segment task counts of every key
// (blockIdx.x = key); key k's prefix lives at segt[key_off[k] + k], n_k + 1 entries
__global__ void jk_seg_prefix_kernel(const long long* const* __restrict__ cnt, const int* __restrict__ key_off,
                                     long long* __restrict__ segt) {
    int k = blockIdx.x;
    int s0 = key_off[k], n = key_off[k + 1] - s0;
    long long* out = segt + s0 + k;
    if (threadIdx.x == 0) {
        long long acc = 0;
        out[0] = 0;
        for (int i = 0; i < n; i++) {
            acc += *cnt[s0 + i];
            out[i + 1] = acc;
        }
    }
}

// J = 2 (V + V^T), K = V + V^T per molecule (blockIdx.y = molecule)
__global__ void jk_symmetrize_batch_kernel(const JKSym* __restrict__ t, double fac) {
    const JKSym m = t[blockIdx.y];
    long long n = (long long)m.nao * m.nao * m.n_dm;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < n;
         e += (long long)gridDim.x * blockDim.x) {
        long long d = e / ((long long)m.nao * m.nao);
        long long r = e - d * m.nao * m.nao;
        int p = (int)(r / m.nao), q = (int)(r % m.nao);
        const double* b = m.in + d * m.nao * m.nao;
        m.out[e] = fac * (b[(size_t)p * m.nao + q] + b[(size_t)q * m.nao + p]);
    }
}

static void free_batch(jk_batch* t) {
    if (!t) return;
    if (t->graph) cudaGraphExecDestroy(t->graph);
    t->fan.destroy();
    cudaFree(t->d_pk);
    cudaFree(t->d_pmol);
    cudaFree(t->d_cq);
    cudaFree(t->d_dmc);
    cudaFree(t->d_seg64);
    cudaFree(t->d_seg32);
    cudaFree(t->d_segt64);
    cudaFree(t->d_segt32);
    cudaFree((void*)t->d_cnt64);
    cudaFree((void*)t->d_cnt32);
    cudaFree(t->d_key_off);
    cudaFree(t->d_work);
    cudaFree(t->d_sym);
    if (t->blas) cublasDestroy(t->blas);
    delete t;
}

static int batch_create(jk_basis_t* const* bases, int nmol, jk_batch* t) {
    BCUDA(cudaGetDevice(&t->device));
    BCUDA(cudaDeviceGetAttribute(&t->nsm, cudaDevAttrMultiProcessorCount, t->device));
    BCUDA(t->fan.init());
    t->nmol = nmol;
    std::vector<JKScreenCQ> cqs;
    std::map<std::tuple<int, int, int>, int> kidx;
    for (int m = 0; m < nmol; m++) {
        jk_basis* b = bases[m];
        if (!b) return jk_internal_set_err(JK_ERR_ARG, "jk_batch_create: null basis");
        if (b->device != t->device) return jk_internal_set_err(JK_ERR_ARG, "jk_batch_create: bases on other devices");
        t->mols.push_back(b);
        t->max_groups = std::max(t->max_groups, b->ngroups);
        for (int c = 0; c < b->ncq; c++) {
            const JKScreenCQ& cq = b->h_cq[c];
            cqs.push_back(cq);
            int cls = jk_internal_class_index(b, cq.cp_ij, cq.cp_kl);
            int np_ij = b->h_group_nprim[cq.gi] * b->h_group_nprim[cq.gj];
            int np_kl = b->h_group_nprim[cq.gk] * b->h_group_nprim[cq.gl];
            auto key = std::make_tuple(cls, np_ij, np_kl);
            auto it = kidx.find(key);
            if (it == kidx.end()) {
                kidx[key] = (int)t->keys.size();
                JKBatchKey k;
                k.cls = cls;
                k.np_ij = np_ij;
                k.np_kl = np_kl;
                t->keys.push_back(k);
                it = kidx.find(key);
            }
            JKBatchKey& k = t->keys[it->second];
            k.segs.push_back({m, c});
            k.max_tasks += cq.cp_ij == cq.cp_kl ? (long long)cq.n_ij * (cq.n_ij + 1) / 2
                                                : (long long)cq.n_ij * cq.n_kl;
        }
    }
    for (auto& k : t->keys)
        if (!jk_internal_batch_launcher(k.cls, 0))
            return jk_internal_set_err(JK_ERR_UNSUPPORTED, "jk_batch_create: class without kernel");
    t->ncq = (int)cqs.size();
    t->key_off.push_back(0);
    std::vector<const long long*> c64, c32;
    for (auto& k : t->keys) {
        for (auto& sgi : k.segs) {
            const JKScreenCQ& cq = t->mols[sgi.first]->h_cq[sgi.second];
            c64.push_back(cq.task0 + 1);
            c32.push_back(cq.task032 + 1);
        }
        t->key_off.push_back(t->key_off.back() + (int)k.segs.size());
    }
    t->nseg = t->key_off.back();
    int nkeys = (int)t->keys.size();
    BCUDA(cudaMalloc(&t->d_cq, sizeof(JKScreenCQ) * std::max(1, t->ncq)));
    if (t->ncq) BCUDA(cudaMemcpy(t->d_cq, cqs.data(), sizeof(JKScreenCQ) * t->ncq, cudaMemcpyHostToDevice));
    BCUDA(cudaMalloc(&t->d_dmc, sizeof(JKDmCond) * nmol));
    BCUDA(cudaMalloc(&t->d_seg64, sizeof(JKSeg) * std::max(1, t->nseg)));
    BCUDA(cudaMalloc(&t->d_seg32, sizeof(JKSeg) * std::max(1, t->nseg)));
    BCUDA(cudaMalloc(&t->d_segt64, sizeof(long long) * (t->nseg + nkeys + 1)));
    BCUDA(cudaMalloc(&t->d_segt32, sizeof(long long) * (t->nseg + nkeys + 1)));
    BCUDA(cudaMalloc((void**)&t->d_cnt64, sizeof(long long*) * std::max(1, t->nseg)));
    BCUDA(cudaMalloc((void**)&t->d_cnt32, sizeof(long long*) * std::max(1, t->nseg)));
    BCUDA(cudaMalloc(&t->d_key_off, sizeof(int) * (nkeys + 1)));
    if (t->nseg) {
        BCUDA(cudaMemcpy((void*)t->d_cnt64, c64.data(), sizeof(long long*) * t->nseg, cudaMemcpyHostToDevice));
        BCUDA(cudaMemcpy((void*)t->d_cnt32, c32.data(), sizeof(long long*) * t->nseg, cudaMemcpyHostToDevice));
    }
    BCUDA(cudaMemcpy(t->d_key_off, t->key_off.data(), sizeof(int) * (nkeys + 1), cudaMemcpyHostToDevice));
    return JK_OK;
}

extern "C" int jk_batch_create(jk_basis_t* const* bases, int nmol, jk_batch_t** out) {
    if (!bases || nmol <= 0 || !out) return jk_internal_set_err(JK_ERR_ARG, "jk_batch_create: invalid arguments");
    jk_batch* t = new jk_batch();
    int rc = batch_create(bases, nmol, t);
    if (rc) {
        free_batch(t);
        *out = nullptr;
        return rc;
    }
    *out = t;
    return JK_OK;
}

extern "C" int jk_batch_destroy(jk_batch_t* t) {
    free_batch(t);
    return JK_OK;
}

// (re)build the segment tables when the density / output buffers change
static int batch_segments(jk_batch* t, const double* const* dms, double* const* vjs, double* const* vks, int n_dm,
                          cudaStream_t st) {
    bool same = t->seg_ndm == n_dm && (int)t->seg_dm.size() == t->nmol;
    for (int m = 0; same && m < t->nmol; m++)
        same = t->seg_dm[m] == dms[m] && t->seg_vj[m] == (vjs ? vjs[m] : nullptr) &&
               t->seg_vk[m] == (vks ? vks[m] : nullptr);
    if (same) return JK_OK;
    // earlier launches may still read the old tables and buffers
    BCUDA(cudaStreamSynchronize(st));
    // pair-packed J side (with J only)
    t->packed = vjs != nullptr;
    std::vector<size_t> dp_off(t->nmol, 0);
    t->pk_max = 0;
    if (t->packed) {
        size_t tot = 0;
        for (int m = 0; m < t->nmol; m++) {
            dp_off[m] = tot;
            tot += (size_t)n_dm * t->mols[m]->pack_total;
            t->pk_max = std::max(t->pk_max, t->mols[m]->pack_total);
        }
        t->pk_jp = tot;
        if (2 * tot > t->pk_cap) {
            cudaFree(t->d_pk);
            t->d_pk = nullptr;
            BCUDA(cudaMalloc(&t->d_pk, sizeof(double) * std::max<size_t>(2 * tot, 1)));
            t->pk_cap = 2 * tot;
        }
        std::vector<JKPackMol> pm(t->nmol);
        for (int m = 0; m < t->nmol; m++) {
            const jk_basis* b = t->mols[m];
            pm[m] = JKPackMol{b->d_pack, b->ncp, b->pack_total, b->d_pair2bra, b->d_pair2ket, b->d_ao_loc,
                              dms[m], b->nao, n_dm, t->d_pk + dp_off[m], t->d_pk + tot + dp_off[m], vjs[m]};
        }
        if (!t->d_pmol) BCUDA(cudaMalloc(&t->d_pmol, sizeof(JKPackMol) * t->nmol));
        BCUDA(cudaMemcpy(t->d_pmol, pm.data(), sizeof(JKPackMol) * t->nmol, cudaMemcpyHostToDevice));
    }
    std::vector<JKSeg> s64(std::max(1, t->nseg)), s32(std::max(1, t->nseg));
    int i = 0;
    for (auto& k : t->keys)
        for (auto& sgi : k.segs) {
            int m = sgi.first;
            jk_internal_fill_seg_batch(t->mols[m], sgi.second, dms[m], n_dm, vjs ? vjs[m] : nullptr,
                                       vks ? vks[m] : nullptr, 0, &s64[i]);
            jk_internal_fill_seg_batch(t->mols[m], sgi.second, dms[m], n_dm, vjs ? vjs[m] : nullptr,
                                       vks ? vks[m] : nullptr, 1, &s32[i]);
            if (t->packed) {
                const jk_basis* b = t->mols[m];
                const JKScreenCQ& cq = b->h_cq[sgi.second];
                const JKPackCls &ki = b->h_pack[cq.cp_ij], &kk = b->h_pack[cq.cp_kl];
                double* dp = t->d_pk + dp_off[m];
                double* jp = t->d_pk + t->pk_jp + dp_off[m];
                for (JKSeg* sg : {&s64[i], &s32[i]}) {
                    sg->dp_ij = dp + ki.off;
                    sg->dp_kl = dp + kk.off;
                    sg->jp_ij = jp + ki.off;
                    sg->jp_kl = jp + kk.off;
                    sg->np_ij = ki.np;
                    sg->np_kl = kk.np;
                    sg->pk_stride = b->pack_total;
                }
            }
            i++;
        }
    t->h_dmc.resize(t->nmol);
    for (int m = 0; m < t->nmol; m++) {
        jk_basis* b = t->mols[m];
        t->h_dmc[m] = JKDmCond{dms[m], b->d_group_ao, b->d_dm_cond, b->nao, n_dm, b->ngroups};
    }
    BCUDA(cudaMemcpy(t->d_seg64, s64.data(), sizeof(JKSeg) * t->nseg, cudaMemcpyHostToDevice));
    BCUDA(cudaMemcpy(t->d_seg32, s32.data(), sizeof(JKSeg) * t->nseg, cudaMemcpyHostToDevice));
    BCUDA(cudaMemcpy(t->d_dmc, t->h_dmc.data(), sizeof(JKDmCond) * t->nmol, cudaMemcpyHostToDevice));
    t->seg_dm.assign(dms, dms + t->nmol);
    t->seg_vj.assign(t->nmol, nullptr);
    t->seg_vk.assign(t->nmol, nullptr);
    for (int m = 0; m < t->nmol; m++) {
        if (vjs) t->seg_vj[m] = vjs[m];
        if (vks) t->seg_vk[m] = vks[m];
    }
    t->seg_ndm = n_dm;
    return JK_OK;
}

extern "C" int jk_batch_build(jk_batch_t* t, const double* const* dms, double* const* vjs, double* const* vks,
                              int n_dm, const jk_opts_t* opts, void* stream) {
    if (!t || !dms || n_dm <= 0) return jk_internal_set_err(JK_ERR_ARG, "jk_batch_build: invalid arguments");
    if (!vjs && !vks) return JK_OK;
    cudaStream_t st = (cudaStream_t)stream;
    int rc = batch_segments(t, dms, vjs, vks, n_dm, st);
    if (rc) return rc;
    double tol = opts ? opts->direct_scf_tol : t->mols[0]->cutoff;
    int nbins = opts && opts->nbins > 0 ? opts->nbins : 10;
    int prescreen = opts ? opts->prescreen : 1;
    double fp32_cutoff = opts ? opts->fp32_cutoff : 0.;
    dim3 g(t->max_groups, t->max_groups, t->nmol);
    jk_dm_cond_batch_kernel<<<g, 256, 0, st>>>(t->d_dmc);
    BCUDA(cudaGetLastError());
    if (t->ncq == 0) return JK_OK;
    rc = jk_internal_screen(t->d_cq, t->ncq, tol, nbins, prescreen, fp32_cutoff, stream);
    if (rc) return rc;
    int nkeys = (int)t->keys.size();
    jk_seg_prefix_kernel<<<nkeys, 32, 0, st>>>(t->d_cnt64, t->d_key_off, t->d_segt64);
    BCUDA(cudaGetLastError());
    if (fp32_cutoff > 0) {
        jk_seg_prefix_kernel<<<nkeys, 32, 0, st>>>(t->d_cnt32, t->d_key_off, t->d_segt32);
        BCUDA(cudaGetLastError());
    }
    if (t->packed) {
        rc = jk_internal_pack_batch(t->d_pmol, t->nmol, t->pk_max, 0, stream);
        if (rc) return rc;
        BCUDA(cudaMemsetAsync(t->d_pk + t->pk_jp, 0, sizeof(double) * t->pk_jp, st));
    }
    BCUDA(t->fan.begin(st));
    for (int k = 0; k < nkeys; k++) {
        const JKBatchKey& key = t->keys[k];
        int off = t->key_off[k], n = t->key_off[k + 1] - off;
        jk_launch_batch_fn f = jk_internal_batch_launcher(key.cls, 0);
        BCUDA(f(t->d_seg64 + off, t->d_segt64 + off + k, n, key.max_tasks, t->nsm, t->fan.pick(2 * k)));
        if (fp32_cutoff > 0) {
            jk_launch_batch_fn f32 = jk_internal_batch_launcher(key.cls, 1);
            if (!f32) return jk_internal_set_err(JK_ERR_UNSUPPORTED, "no FP32 kernel for a class");
            BCUDA(f32(t->d_seg32 + off, t->d_segt32 + off + k, n, key.max_tasks, t->nsm, t->fan.pick(2 * k + 1)));
        }
    }
    BCUDA(t->fan.end(st));
    if (t->packed) {
        rc = jk_internal_pack_batch(t->d_pmol, t->nmol, t->pk_max, 1, stream);
        if (rc) return rc;
    }
    return JK_OK;
}

static cublasStatus_t gemm_rm_b(cublasHandle_t h, bool ta, bool tb, int M, int N, int K, const double* A, int lda,
                                const double* B, int ldb, double* C, int ldc) {
    const double one = 1.0, zero = 0.0;
    return cublasDgemm(h, tb ? CUBLAS_OP_T : CUBLAS_OP_N, ta ? CUBLAS_OP_T : CUBLAS_OP_N, N, M, K, &one, B, ldb, A,
                       lda, &zero, C, ldc);
}

#define BBLAS(x)                                                                           \
    do {                                                                                   \
        if ((x) != CUBLAS_STATUS_SUCCESS) return jk_internal_set_err(JK_ERR_CUDA, #x);     \
    } while (0)

// Full J/K of every molecule in its own basis: dms_m = C_m D_m C_m^T, one
// batched build, then J_m = 2 C_m^T (V + V^T) C_m, K_m = C_m^T (V + V^T) C_m.
// coeffs[m] (nao_m, nao0s[m]) row-major device; dm0s/vj0s/vk0s device
// (n_dm, nao0, nao0); vj0s/vk0s overwritten (either may be NULL).
extern "C" int jk_batch_get_jk(jk_batch_t* t, const double* const* coeffs, const int* nao0s,
                               const double* const* dm0s, double* const* vj0s, double* const* vk0s, int n_dm,
                               const jk_opts_t* opts, void* stream) {
    if (!t || !coeffs || !nao0s || !dm0s || n_dm <= 0)
        return jk_internal_set_err(JK_ERR_ARG, "jk_batch_get_jk: invalid arguments");
    cudaStream_t st = (cudaStream_t)stream;
    int nmol = t->nmol;
    if (t->w_ndm != n_dm) {
        size_t off = 0;
        t->w_dms.resize(nmol);
        t->w_vj.resize(nmol);
        t->w_vk.resize(nmol);
        t->w_sym.resize(nmol);
        t->w_tmp.resize(nmol);
        for (int m = 0; m < nmol; m++) {
            size_t nn = (size_t)t->mols[m]->nao * t->mols[m]->nao * n_dm;
            t->w_dms[m] = off;
            off += nn;
            t->w_vj[m] = off;
            off += nn;
            t->w_vk[m] = off;
            off += nn;
            t->w_sym[m] = off;
            off += nn;
            t->w_tmp[m] = off;
            off += (size_t)t->mols[m]->nao * nao0s[m];
        }
        BCUDA(cudaStreamSynchronize(st));
        cudaFree(t->d_work);
        t->d_work = nullptr;
        BCUDA(cudaMalloc(&t->d_work, sizeof(double) * std::max<size_t>(off, 1)));
        t->work_cap = off;
        cudaFree(t->d_sym);
        t->d_sym = nullptr;
        // symmetrisation tables: J inputs in [0, nmol), K inputs in [nmol, 2 nmol)
        BCUDA(cudaMalloc(&t->d_sym, sizeof(JKSym) * 2 * nmol));
        std::vector<JKSym> sy(2 * nmol);
        for (int m = 0; m < nmol; m++) {
            sy[m] = JKSym{t->d_work + t->w_vj[m], t->d_work + t->w_sym[m], t->mols[m]->nao, n_dm};
            sy[nmol + m] = JKSym{t->d_work + t->w_vk[m], t->d_work + t->w_sym[m], t->mols[m]->nao, n_dm};
        }
        BCUDA(cudaMemcpy(t->d_sym, sy.data(), sizeof(JKSym) * 2 * nmol, cudaMemcpyHostToDevice));
        t->w_ndm = n_dm;
    }
    if (!t->blas) BBLAS(cublasCreate(&t->blas));
    BBLAS(cublasSetStream(t->blas, st));
    std::vector<const double*> dms(nmol);
    std::vector<double*> vjs(nmol), vks(nmol);
    for (int m = 0; m < nmol; m++) {
        jk_basis* b = t->mols[m];
        int nao = b->nao, nao0 = nao0s[m];
        double* w = t->d_work;
        for (int d = 0; d < n_dm; d++) {
            BBLAS(gemm_rm_b(t->blas, false, false, nao, nao0, nao0, coeffs[m], nao0,
                            dm0s[m] + (size_t)d * nao0 * nao0, nao0, w + t->w_tmp[m], nao0));
            BBLAS(gemm_rm_b(t->blas, false, true, nao, nao, nao0, w + t->w_tmp[m], nao0, coeffs[m], nao0,
                            w + t->w_dms[m] + (size_t)d * nao * nao, nao));
        }
        size_t nn = (size_t)nao * nao * n_dm;
        if (vj0s) BCUDA(cudaMemsetAsync(w + t->w_vj[m], 0, sizeof(double) * nn, st));
        if (vk0s) BCUDA(cudaMemsetAsync(w + t->w_vk[m], 0, sizeof(double) * nn, st));
        dms[m] = w + t->w_dms[m];
        vjs[m] = w + t->w_vj[m];
        vks[m] = w + t->w_vk[m];
    }
    int rc = jk_batch_build(t, dms.data(), vj0s ? vjs.data() : nullptr, vk0s ? vks.data() : nullptr, n_dm, opts,
                            stream);
    if (rc) return rc;
    for (int pass = 0; pass < 2; pass++) {
        double* const* outs = pass == 0 ? vj0s : vk0s;
        if (!outs) continue;
        dim3 g(32, nmol);
        jk_symmetrize_batch_kernel<<<g, 256, 0, st>>>(t->d_sym + (pass == 0 ? 0 : nmol), pass == 0 ? 2.0 : 1.0);
        BCUDA(cudaGetLastError());
        for (int m = 0; m < nmol; m++) {
            jk_basis* b = t->mols[m];
            int nao = b->nao, nao0 = nao0s[m];
            double* w = t->d_work;
            for (int d = 0; d < n_dm; d++) {
                BBLAS(gemm_rm_b(t->blas, false, false, nao, nao0, nao, w + t->w_sym[m] + (size_t)d * nao * nao, nao,
                                coeffs[m], nao0, w + t->w_tmp[m], nao0));
                BBLAS(gemm_rm_b(t->blas, true, false, nao0, nao0, nao, coeffs[m], nao0, w + t->w_tmp[m], nao0,
                                outs[m] + (size_t)d * nao0 * nao0, nao0));
            }
        }
    }
    return JK_OK;
}
