// Batched J/K builds: many molecules (one jk_basis each) in one pass.
//
// The single-molecule path launches one kernel per class quartet; for small
// molecules those launches are tiny and the GPU idles between them.  Here the
// class quartets of all molecules that share a class key become segments of
// ONE launch, so a batch of hundreds of molecules costs one launch per class
// key plus three bookkeeping launches (density condensation, screening,
// segment prefixes), with no host synchronisation; the whole sequence can be
// captured into a CUDA graph and replayed every SCF iteration.  A key is the
// class (four angular momenta), plus the two primitive counts for the team
// kernels, whose blocks loop over the primitives in step.  Within a key the
// segments are ordered by descending task count, so the largest molecules'
// work is handed out first.
//
// Class quartets with at least `solo_tasks` unscreened tasks are not merged:
// each runs as its own launch of the single-molecule kernel (segment in the
// parameter bank, as jk_build launches it), in molecule order, fanned out
// over the side streams ahead of the merged keys.  Such a launch fills the
// device by itself, and merging it costs more than it saves (measured on
// 6-31G* molecules of 276-588 functions: 13-36 % slower merged, while
// molecules below 160 functions build 4.7x faster merged).
//
// Launch shape per key (JKBatchCfg): static contiguous chunks, or the
// persistent mode in which a grid of the device's resident capacity takes
// chunks from a device counter.  jk_batch_tune times the candidate shapes of
// every key on the batch itself and keeps the fastest; its choices can be
// written to and read from a cache file.
#include <math.h>
#include <stdio.h>
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
    int cls, np_ij, np_kl;                  // np_* = -1: any primitive count
    std::vector<std::pair<int, int>> segs;  // (molecule, class quartet)
    std::vector<long long> seg_tasks;       // unscreened tasks of each segment
    long long max_tasks = 0;
    JKBatchCfg cfg[2] = {{nullptr, 0, 1}, {nullptr, 0, 1}};  // FP64 part, FP32 part (queue set at launch)
    float tuned_ms[2] = {-1.f, -1.f};
};

// a class quartet launched on its own (see the top of the file)
struct JKSolo {
    int mol, cq, cls;
    long long tasks;  // unscreened
    JKSeg s64, s32;   // FP64 and FP32 parts, filled with the segment tables
};

struct jk_batch {
    int device = 0, nsm = 148, nmol = 0, max_groups = 0;
    long long solo_tasks = JK_BATCH_SOLO_TASKS;
    std::vector<jk_basis*> mols;
    std::vector<JKBatchKey> keys;
    std::vector<JKSolo> solo;
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
    unsigned long long* d_queue = nullptr;  // 2 work counters per key (persistent launches)
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
    cudaFree(t->d_queue);
    cudaFree(t->d_work);
    cudaFree(t->d_sym);
    if (t->blas) cublasDestroy(t->blas);
    delete t;
}

static int batch_create(jk_basis_t* const* bases, int nmol, long long solo_tasks, jk_batch* t) {
    t->solo_tasks = solo_tasks;
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
            const long long n = cq.cp_ij == cq.cp_kl ? (long long)cq.n_ij * (cq.n_ij + 1) / 2
                                                     : (long long)cq.n_ij * cq.n_kl;
            if (solo_tasks > 0 && n >= solo_tasks) {
                JKSolo so{};
                so.mol = m;
                so.cq = c;
                so.cls = cls;
                so.tasks = n;
                t->solo.push_back(so);
                continue;
            }
            int np_ij = b->h_group_nprim[cq.gi] * b->h_group_nprim[cq.gj];
            int np_kl = b->h_group_nprim[cq.gk] * b->h_group_nprim[cq.gl];
            if (!jk_internal_class_team(cls)) np_ij = np_kl = -1;
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
            k.seg_tasks.push_back(n);
            k.max_tasks += n;
        }
    }
    // longest first within every key (stable: ties keep molecule order)
    for (auto& k : t->keys) {
        std::vector<int> ord(k.segs.size());
        for (size_t i = 0; i < ord.size(); i++) ord[i] = (int)i;
        std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return k.seg_tasks[a] > k.seg_tasks[b]; });
        std::vector<std::pair<int, int>> segs(ord.size());
        std::vector<long long> tasks(ord.size());
        for (size_t i = 0; i < ord.size(); i++) {
            segs[i] = k.segs[ord[i]];
            tasks[i] = k.seg_tasks[ord[i]];
        }
        k.segs.swap(segs);
        k.seg_tasks.swap(tasks);
    }
    for (auto& k : t->keys)
        if (!jk_internal_batch_launcher(k.cls, 0))
            return jk_internal_set_err(JK_ERR_UNSUPPORTED, "jk_batch_create: class without kernel");
    for (auto& so : t->solo)
        if (!jk_internal_batch_launcher(so.cls, 0))
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
    BCUDA(cudaMalloc(&t->d_queue, sizeof(unsigned long long) * 2 * std::max(1, nkeys)));
    if (t->nseg) {
        BCUDA(cudaMemcpy((void*)t->d_cnt64, c64.data(), sizeof(long long*) * t->nseg, cudaMemcpyHostToDevice));
        BCUDA(cudaMemcpy((void*)t->d_cnt32, c32.data(), sizeof(long long*) * t->nseg, cudaMemcpyHostToDevice));
    }
    BCUDA(cudaMemcpy(t->d_key_off, t->key_off.data(), sizeof(int) * (nkeys + 1), cudaMemcpyHostToDevice));
    return JK_OK;
}

extern "C" int jk_batch_create_ex(jk_basis_t* const* bases, int nmol, long long solo_tasks, jk_batch_t** out) {
    if (!bases || nmol <= 0 || !out) return jk_internal_set_err(JK_ERR_ARG, "jk_batch_create: invalid arguments");
    jk_batch* t = new jk_batch();
    int rc = batch_create(bases, nmol, solo_tasks, t);
    if (rc) {
        free_batch(t);
        *out = nullptr;
        return rc;
    }
    *out = t;
    return JK_OK;
}

extern "C" int jk_batch_create(jk_basis_t* const* bases, int nmol, jk_batch_t** out) {
    return jk_batch_create_ex(bases, nmol, JK_BATCH_SOLO_TASKS, out);
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
    // pair-packed J side of molecule m's class quartet c in both parts
    auto set_packed = [&](int m, int c, JKSeg* a, JKSeg* b2) {
        if (!t->packed) return;
        const jk_basis* b = t->mols[m];
        const JKScreenCQ& cq = b->h_cq[c];
        const JKPackCls &ki = b->h_pack[cq.cp_ij], &kk = b->h_pack[cq.cp_kl];
        double* dp = t->d_pk + dp_off[m];
        double* jp = t->d_pk + t->pk_jp + dp_off[m];
        for (JKSeg* sg : {a, b2}) {
            sg->dp_ij = dp + ki.off;
            sg->dp_kl = dp + kk.off;
            sg->jp_ij = jp + ki.off;
            sg->jp_kl = jp + kk.off;
            sg->np_ij = ki.np;
            sg->np_kl = kk.np;
            sg->pk_stride = b->pack_total;
        }
    };
    for (auto& so : t->solo) {
        const int m = so.mol;
        jk_internal_fill_seg_batch(t->mols[m], so.cq, dms[m], n_dm, vjs ? vjs[m] : nullptr, vks ? vks[m] : nullptr, 0,
                                   &so.s64);
        jk_internal_fill_seg_batch(t->mols[m], so.cq, dms[m], n_dm, vjs ? vjs[m] : nullptr, vks ? vks[m] : nullptr, 1,
                                   &so.s32);
        set_packed(m, so.cq, &so.s64, &so.s32);
    }
    std::vector<JKSeg> s64(std::max(1, t->nseg)), s32(std::max(1, t->nseg));
    int i = 0;
    for (auto& k : t->keys) {
        for (auto& sgi : k.segs) {
            int m = sgi.first;
            jk_internal_fill_seg_batch(t->mols[m], sgi.second, dms[m], n_dm, vjs ? vjs[m] : nullptr,
                                       vks ? vks[m] : nullptr, 0, &s64[i]);
            jk_internal_fill_seg_batch(t->mols[m], sgi.second, dms[m], n_dm, vjs ? vjs[m] : nullptr,
                                       vks ? vks[m] : nullptr, 1, &s32[i]);
            set_packed(m, sgi.second, &s64[i], &s32[i]);
            i++;
        }
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

// everything before the class launches: segment tables, density
// condensation, screening, task prefixes, pair-packed densities
static int batch_prepare(jk_batch* t, const double* const* dms, double* const* vjs, double* const* vks, int n_dm,
                         const jk_opts_t* opts, cudaStream_t st) {
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
    rc = jk_internal_screen(t->d_cq, t->ncq, tol, nbins, prescreen, fp32_cutoff, st);
    if (rc) return rc;
    int nkeys = (int)t->keys.size();
    if (nkeys > 0) {
        jk_seg_prefix_kernel<<<nkeys, 32, 0, st>>>(t->d_cnt64, t->d_key_off, t->d_segt64);
        BCUDA(cudaGetLastError());
    }
    if (fp32_cutoff > 0 && nkeys > 0) {
        jk_seg_prefix_kernel<<<nkeys, 32, 0, st>>>(t->d_cnt32, t->d_key_off, t->d_segt32);
        BCUDA(cudaGetLastError());
    }
    if (t->packed) {
        rc = jk_internal_pack_batch(t->d_pmol, t->nmol, t->pk_max, 0, st);
        if (rc) return rc;
        BCUDA(cudaMemsetAsync(t->d_pk + t->pk_jp, 0, sizeof(double) * t->pk_jp, st));
    }
    return JK_OK;
}

// the class launch of key k, part 0 (FP64) or 1 (FP32), with shape cfg
static int batch_launch_key(jk_batch* t, int k, int part, const JKBatchCfg& cfg, cudaStream_t st) {
    const JKBatchKey& key = t->keys[k];
    int off = t->key_off[k], n = t->key_off[k + 1] - off;
    jk_launch_batch_fn f = jk_internal_batch_launcher(key.cls, part);
    if (!f) return jk_internal_set_err(JK_ERR_UNSUPPORTED, "no kernel for a class of the batch");
    JKBatchCfg c = cfg;
    if (c.grab > 0) c.queue = t->d_queue + 2 * k + part;
    else c.queue = nullptr;
    const JKSeg* segs = (part ? t->d_seg32 : t->d_seg64) + off;
    const long long* segt = (part ? t->d_segt32 : t->d_segt64) + off + k;
    BCUDA(f(segs, segt, n, key.max_tasks, t->nsm, c, st));
    return JK_OK;
}

extern "C" int jk_batch_build(jk_batch_t* t, const double* const* dms, double* const* vjs, double* const* vks,
                              int n_dm, const jk_opts_t* opts, void* stream) {
    if (!t || !dms || n_dm <= 0) return jk_internal_set_err(JK_ERR_ARG, "jk_batch_build: invalid arguments");
    if (!vjs && !vks) return JK_OK;
    cudaStream_t st = (cudaStream_t)stream;
    int rc = batch_prepare(t, dms, vjs, vks, n_dm, opts, st);
    if (rc || t->ncq == 0) return rc;
    const bool mixed = opts && opts->fp32_cutoff > 0;
    int nkeys = (int)t->keys.size();
    // work counters of the persistent launches start at zero every build
    BCUDA(cudaMemsetAsync(t->d_queue, 0, sizeof(unsigned long long) * 2 * nkeys, st));
    BCUDA(t->fan.begin(st));
    int lane = 0;  // FP64 parts on the even side streams, FP32 parts on the odd ones
    for (const JKSolo& so : t->solo) {
        const JKScreenCQ& cq = t->mols[so.mol]->h_cq[so.cq];
        rc = jk_internal_launch_part(so.cls, 0, so.s64, cq.task0, so.tasks, t->nsm, t->fan.pick(2 * lane));
        if (rc) return rc;
        if (mixed) {
            rc = jk_internal_launch_part(so.cls, 1, so.s32, cq.task032, so.tasks, t->nsm, t->fan.pick(2 * lane + 1));
            if (rc) return rc;
        }
        lane++;
    }
    for (int k = 0; k < nkeys; k++, lane++) {
        rc = batch_launch_key(t, k, 0, t->keys[k].cfg[0], t->fan.pick(2 * lane));
        if (rc) return rc;
        if (mixed) {
            rc = batch_launch_key(t, k, 1, t->keys[k].cfg[1], t->fan.pick(2 * lane + 1));
            if (rc) return rc;
        }
    }
    BCUDA(t->fan.end(st));
    if (t->packed) {
        rc = jk_internal_pack_batch(t->d_pmol, t->nmol, t->pk_max, 1, stream);
        if (rc) return rc;
    }
    return JK_OK;
}

// ---------------------------------------------------------------------------
// Autotuner.  For every key (and both parts in the mixed mode) the candidate
// launch shapes are timed on this batch with CUDA events, each launch alone
// on the caller's stream after the bookkeeping of a real build, and the
// fastest is kept.  Candidates: static chunks; the persistent mode at one
// resident grid with three grab sizes (tasks per warp for the thread
// kernels, per team for the team kernels, per block for the generic kernel)
// and at two resident grids with the middle one.  A cache file keeps the
// choices per (class, primitive counts, part, log2 of the task count); keys
// found there are not timed again.
// ---------------------------------------------------------------------------
static bool class_is_generic(int cls) {
    const int ll = cls % 7, lk = (cls / 7) % 7, lj = (cls / 49) % 7, li = cls / 343;
    return li > JK_LMAX || lj > JK_LMAX || lk > JK_LMAX || ll > JK_LMAX;
}

static int cand_grabs(int cls, int* g) {
    if (jk_internal_class_team(cls)) { g[0] = 2; g[1] = 8; g[2] = 32; }
    else if (class_is_generic(cls)) { g[0] = 1; g[1] = 4; g[2] = 16; }
    else { g[0] = 64; g[1] = 256; g[2] = 1024; }
    return 3;
}

static std::string tune_key_str(const JKBatchKey& k, int part) {
    int b = 0;
    for (long long x = k.max_tasks; x > 1; x >>= 1) b++;
    char buf[96];
    snprintf(buf, sizeof(buf), "%d %d %d %d %d", k.cls, k.np_ij, k.np_kl, part, b);
    return buf;
}

extern "C" int jk_batch_tune(jk_batch_t* t, const double* const* dms, double* const* vjs, double* const* vks,
                             int n_dm, const jk_opts_t* opts, const char* cache_path, void* stream) {
    if (!t || !dms || n_dm <= 0 || (!vjs && !vks))
        return jk_internal_set_err(JK_ERR_ARG, "jk_batch_tune: invalid arguments");
    cudaStream_t st = (cudaStream_t)stream;
    int nkeys = (int)t->keys.size();
    const bool mixed = opts && opts->fp32_cutoff > 0;
    // cached choices: "cls np_ij np_kl part log2tasks mode grab grid_mul ms"
    std::map<std::string, std::pair<JKBatchCfg, float>> cache;
    if (cache_path) {
        FILE* f = fopen(cache_path, "r");
        if (f) {
            char line[256];
            while (fgets(line, sizeof(line), f)) {
                int cls, a, b, part, lg, grab, gm;
                float ms;
                if (sscanf(line, "%d %d %d %d %d %d %d %f", &cls, &a, &b, &part, &lg, &grab, &gm, &ms) != 8) continue;
                char key[96];
                snprintf(key, sizeof(key), "%d %d %d %d %d", cls, a, b, part, lg);
                cache[key] = {JKBatchCfg{nullptr, grab, gm}, ms};
            }
            fclose(f);
        }
    }
    int rc = batch_prepare(t, dms, vjs, vks, n_dm, opts, st);
    if (rc) return rc;
    cudaEvent_t e0, e1;
    BCUDA(cudaEventCreate(&e0));
    BCUDA(cudaEventCreate(&e1));
    for (int k = 0; k < nkeys && t->ncq; k++) {
        JKBatchKey& key = t->keys[k];
        for (int part = 0; part < (mixed ? 2 : 1); part++) {
            const std::string ks = tune_key_str(key, part);
            auto hit = cache.find(ks);
            if (hit != cache.end()) {
                key.cfg[part] = hit->second.first;
                key.tuned_ms[part] = hit->second.second;
                continue;
            }
            int g[3];
            cand_grabs(key.cls, g);
            std::vector<JKBatchCfg> cands = {{nullptr, 0, 1}};
            for (int i = 0; i < 3; i++) cands.push_back({nullptr, g[i], 1});
            cands.push_back({nullptr, g[1], 2});
            // untimed first launch (attributes, instruction cache)
            BCUDA(cudaMemsetAsync(t->d_queue, 0, sizeof(unsigned long long) * 2 * nkeys, st));
            rc = batch_launch_key(t, k, part, cands[0], st);
            if (rc) return rc;
            float best = -1.f;
            for (const JKBatchCfg& c : cands) {
                float tmin = -1.f;
                for (int rep = 0; rep < 1; rep++) {
                    BCUDA(cudaMemsetAsync(t->d_queue, 0, sizeof(unsigned long long) * 2 * nkeys, st));
                    BCUDA(cudaEventRecord(e0, st));
                    rc = batch_launch_key(t, k, part, c, st);
                    if (rc) return rc;
                    BCUDA(cudaEventRecord(e1, st));
                    BCUDA(cudaEventSynchronize(e1));
                    float ms = 0.f;
                    BCUDA(cudaEventElapsedTime(&ms, e0, e1));
                    if (tmin < 0 || ms < tmin) tmin = ms;
                }
                if (best < 0 || tmin < best) {
                    best = tmin;
                    key.cfg[part] = c;
                }
            }
            key.tuned_ms[part] = best;
            cache[ks] = {key.cfg[part], best};
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    BCUDA(cudaStreamSynchronize(st));
    // the timing runs accumulated into the outputs: clear them
    for (int m = 0; m < t->nmol; m++) {
        size_t nn = (size_t)t->mols[m]->nao * t->mols[m]->nao * n_dm;
        if (vjs && vjs[m]) BCUDA(cudaMemset(vjs[m], 0, sizeof(double) * nn));
        if (vks && vks[m]) BCUDA(cudaMemset(vks[m], 0, sizeof(double) * nn));
    }
    if (cache_path) {
        FILE* f = fopen(cache_path, "w");
        if (!f) return jk_internal_set_err(JK_ERR_ARG, "jk_batch_tune: cannot write the cache file");
        fprintf(f, "# byteqc_b200 batch launch shapes: cls np_ij np_kl part log2tasks grab grid_mul ms\n");
        for (auto& kv : cache)
            fprintf(f, "%s %d %d %.4f\n", kv.first.c_str(), kv.second.first.grab, kv.second.first.grid_mul,
                    kv.second.second);
        fclose(f);
    }
    return JK_OK;
}

extern "C" int jk_batch_nsolo(const jk_batch_t* t, int* nsolo) {
    if (!t || !nsolo) return jk_internal_set_err(JK_ERR_ARG, "jk_batch_nsolo: invalid arguments");
    *nsolo = (int)t->solo.size();
    return JK_OK;
}

// launch shapes chosen for the batch: per key cls, np_ij, np_kl, then for
// parts 0 and 1 grab, grid_mul and the tuned time in microseconds (-1 if
// not tuned); out holds 12 ints per key
extern "C" int jk_batch_info(const jk_batch_t* t, int* nkeys, int* out) {
    if (!t || !nkeys) return jk_internal_set_err(JK_ERR_ARG, "jk_batch_info: invalid arguments");
    *nkeys = (int)t->keys.size();
    if (!out) return JK_OK;
    for (size_t k = 0; k < t->keys.size(); k++) {
        const JKBatchKey& key = t->keys[k];
        int* o = out + 12 * k;
        o[0] = key.cls;
        o[1] = key.np_ij;
        o[2] = key.np_kl;
        o[3] = (int)std::min<long long>(key.max_tasks, 2147483647LL);
        for (int p = 0; p < 2; p++) {
            o[4 + 4 * p] = key.cfg[p].grab;
            o[5 + 4 * p] = key.cfg[p].grid_mul;
            o[6 + 4 * p] = (int)(key.tuned_ms[p] * 1000.f);
            o[7 + 4 * p] = (int)key.segs.size();
        }
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
