// Internal helpers of jk_host.cu shared with other translation units of
// libjk.so (not part of the C-ABI).
#pragma once
#include <cublas_v2.h>

#include <string>
#include <vector>

#include "jk_common.cuh"
#include "../../include/byteqc_jk.h"

// One class quartet (cp_ij >= cp_kl) of one basis, as the screening kernel
// sees it: pair counts, group indices and the device buffers it reads/writes.
struct JKScreenCQ {
    int cp_ij, cp_kl;
    int gi, gj, gk, gl;
    int n_ij, n_kl;
    int ngroups;
    const double *lq_ij, *lq_kl;  // clipped log q of the two classes
    const double *rq_ij, *rq_kl;  // unclipped log q (mixed-precision split)
    const double* dm_cond;        // ngroups x ngroups
    long long *qoff, *qoff32;     // row prefixes, FP64 and FP32 parts
    int* klb;                     // first FP32 column per row
    long long *task0, *task032;   // {0, count} of each part
    // host bookkeeping
    int pair_ij0, pair_kl0;
    long long qoff_off;
};


int jk_internal_set_err(int code, const char* msg);
// pair counts of the two classes and the working-basis size
int jk_internal_class_info(const jk_basis_t* b, int cp_ij, int cp_kl, int* n_ij, int* n_kl, int* nao);
void jk_internal_fill_seg(const jk_basis_t* b, int cp_ij, int cp_kl, const long long* qoff, int n_ij,
                          const double* dm, int n_dm, double* vj, double* vk, JKSeg* out);
// launch the class kernel of (cp_ij, cp_kl) on a device segment table of one entry
int jk_internal_launch(const jk_basis_t* b, int cp_ij, int cp_kl, const JKSeg& seg, const long long* d_task0,
                       long long max_tasks, void* stream);

// Side streams of the class launches.  Every class kernel adds into J and K
// with atomics, so launches of different class quartets (and the FP64 and
// FP32 parts of one) may run concurrently; spreading them over a few
// streams overlaps the ramp-up and tail of the many small launches of a
// build.  begin() forks from the caller's stream with an event, end() joins
// back (both record into a CUDA graph when the caller's stream is captured).
#define JK_SIDE_STREAMS 8
struct JKFanout {
    cudaStream_t s[JK_SIDE_STREAMS] = {};
    cudaEvent_t fork = nullptr;
    cudaEvent_t join[JK_SIDE_STREAMS] = {};
    cudaError_t init() {
        cudaError_t e = cudaEventCreateWithFlags(&fork, cudaEventDisableTiming);
        for (int i = 0; e == cudaSuccess && i < JK_SIDE_STREAMS; i++) {
            e = cudaStreamCreateWithFlags(&s[i], cudaStreamNonBlocking);
            if (e == cudaSuccess) e = cudaEventCreateWithFlags(&join[i], cudaEventDisableTiming);
        }
        return e;
    }
    cudaError_t begin(cudaStream_t st) {
        cudaError_t e = cudaEventRecord(fork, st);
        for (int i = 0; e == cudaSuccess && i < JK_SIDE_STREAMS; i++) e = cudaStreamWaitEvent(s[i], fork, 0);
        return e;
    }
    cudaStream_t pick(int i) const { return s[i % JK_SIDE_STREAMS]; }
    cudaError_t end(cudaStream_t st) {
        cudaError_t e = cudaSuccess;
        for (int i = 0; e == cudaSuccess && i < JK_SIDE_STREAMS; i++) {
            e = cudaEventRecord(join[i], s[i]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(st, join[i], 0);
        }
        return e;
    }
    void destroy() {
        for (int i = 0; i < JK_SIDE_STREAMS; i++) {
            if (s[i]) cudaStreamDestroy(s[i]);
            if (join[i]) cudaEventDestroy(join[i]);
            s[i] = nullptr;
            join[i] = nullptr;
        }
        if (fork) cudaEventDestroy(fork);
        fork = nullptr;
    }
};

// one class pair in the pair-packed density / J buffers of jk_build
struct JKPackCls {
    long long off;      // first packed element of the class
    int np, nfi, nfj;   // pairs, Cartesian components of the two shells
    int pair0;          // first pair of the class
};

// one molecule of a batched pack / unpack of the pair-packed J side
struct JKPackMol {
    const JKPackCls* cls;
    int ncls;
    long long total;
    const int *pair2bra, *pair2ket, *ao_loc;
    const double* dm;
    int nao, n_dm;
    double* dp;        // mode 0 output
    const double* jp;  // mode 1 input
    double* vj;        // mode 1 output
};

// Per-geometry state (opaque to callers of the C-ABI)
struct jk_basis {
    // class quartets and their screening records
    int device = 0, nsm = 148;
    const double* rys = nullptr;  // shared per-device Rys table
    int natm = 0, nbas = 0, nao = 0, ngroups = 0, ncp = 0, ncq = 0;
    double diag_fac = 0.5, cutoff = 1e-13;
    std::vector<int> h_ao_loc, h_group_off, h_group_l, h_group_nprim;
    std::vector<int> h_cls_gi, h_cls_gj, h_pair_locs, h_prim_locs, h_pair2bra, h_pair2ket;
    std::vector<double> h_log_q, h_log_q_raw, h_qcond;
    std::vector<JKScreenCQ> h_cq;
    std::vector<double> h_cq_cost;     // unscreened work of each class quartet (shard plans)
    std::vector<int> h_cq_owner;       // owner of each class quartet in the plan of
    int cq_owner_n = 0;                // cq_owner_n shards
    std::vector<long long> h_qoff_off;
    long long qoff_total = 0;
    // device
    int *d_atm = nullptr, *d_bas = nullptr, *d_ao_loc = nullptr, *d_group_ao = nullptr;
    double *d_env = nullptr, *d_bas_x = nullptr, *d_qcond = nullptr;
    int *d_pair2bra = nullptr, *d_pair2ket = nullptr;
    double *d_log_q = nullptr, *d_log_q_raw = nullptr, *d_prim = nullptr;  // prim: a12|e12|x12|y12|z12|1/a12
    float* d_primf = nullptr;  // FP32 path: a12|1/a12|e12/a12|P-R_bra (x, y, z)
    long long nprim_total = 0;
    JKScreenCQ* d_cq = nullptr;
    long long *d_qoff = nullptr, *d_task0 = nullptr;
    long long *d_qoff32 = nullptr, *d_task032 = nullptr;  // FP32 part of the mixed mode
    int* d_klb = nullptr;
    double* d_dm_cond = nullptr;
    // reference-compatible single class-pair path
    long long* d_qoff1 = nullptr;
    long long* d_task01 = nullptr;
    long long qoff1_cap = 0;
    JKFanout fan;  // side streams of the class launches
    double* d_pgeo = nullptr;  // pair geometry (JKSeg::pgeo)
    std::vector<int> h_pnp;    // primitive pairs above the exponent cutoff, per pair
    int* d_pnp = nullptr;
    int* d_pao = nullptr;      // first AOs of the pair's shells (JKSeg::pao)
    // pair-packed J side of jk_build
    std::vector<JKPackCls> h_pack;
    JKPackCls* d_pack = nullptr;
    long long pack_total = 0;  // packed elements per density
    double* d_pk = nullptr;    // n_dm x pack_total densities, then as many J accumulators
    size_t pk_cap = 0;
    // transform workspace
    cublasHandle_t blas = nullptr;
    double* d_work = nullptr;
    size_t work_cap = 0;
};

// launch one class quartet of basis b as a single segment
int jk_internal_class_index(const jk_basis_t* b, int cp_ij, int cp_kl);
// the single-segment launch of a class (FP64 part or FP32 part), as jk_build makes it
int jk_internal_launch_part(int class_idx, int fp32, const JKSeg& seg, const long long* d_task0, long long max_tasks,
                            int nsm, void* stream);
jk_launch_batch_fn jk_internal_batch_launcher(int class_idx, int fp32);
// 1 if the class runs a team kernel (one primitive count per launch)
int jk_internal_class_team(int class_idx);
void jk_internal_fill_seg_batch(const jk_basis_t* b, int c, const double* dm, int n_dm, double* vj, double* vk,
                                int fp32, JKSeg* out);
// pack (mode 0) or unpack (mode 1) the J side of nmol molecules (device table)
int jk_internal_pack_batch(const JKPackMol* d_mols, int nmol, long long max_total, int mode, void* stream);
int jk_internal_screen(const JKScreenCQ* d_cq, int ncq, double tol, int nbins, int prescreen, double fp32_cutoff,
                       void* stream);
