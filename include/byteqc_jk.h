/*
 * byteqc_jk.h -- C-ABI of the B200 direct-SCF J/K engine (libjk.so).
 *
 * Drop-in boundary for the reference's ctypes interface of ByteQC cuobc's J/K
 * path (cuobc/lib/__init__.py:39-42 loads libgint/libgvhf; the Python side is
 * cuobc/scf/hf.py).  All functions return an int status (JK_OK on success)
 * and never exit the process; jk_last_error() describes the last failure of
 * the calling thread.  Device pointers are plain CUDA device addresses;
 * `stream` is a cudaStream_t passed as void* (NULL = legacy default stream).
 *
 * Working basis: the decontracted Cartesian basis with shells sorted into
 * groups of equal (l, nprim), exactly as the reference's _VHFOpt.build
 * prepares it (cuobc/scf/hf.py:288-330, 481-564).  Angular momentum up to h
 * (l = 5), as the reference's GPU kernels.  The J/K entries need the groups
 * in increasing l (classes out of that order report JK_ERR_UNSUPPORTED);
 * jk_fill_int2e takes them in any order (the density-fitting basis of
 * cuobc/lib/int3c.py:208-264 appends an exponent-0 s shell and the
 * auxiliary basis after the molecule's shells).
 */
#ifndef BYTEQC_JK_H
#define BYTEQC_JK_H

#ifdef __cplusplus
extern "C" {
#endif

#define JK_OK 0
#define JK_ERR_CUDA 1        /* CUDA / cuBLAS failure (launch, copy, OOM) */
#define JK_ERR_UNSUPPORTED 2 /* angular momentum or class not handled */
#define JK_ERR_ARG 3         /* invalid argument */

typedef struct jk_basis jk_basis_t;
typedef struct jk_batch jk_batch_t;

typedef struct {
    double direct_scf_tol; /* density screen threshold (mf.direct_scf_tol)    */
    int nbins;             /* log-Schwarz bins (hf.py:96-100: max(10, ...))    */
    int prescreen;         /* class-level density screen on/off (hf.py:139)   */
    double fp32_cutoff;    /* mixed precision: FP32 recursion below this bound;
                              0 disables                                       */
    int shard;             /* sharded builds (one GPU per rank): this rank's  */
    int nshards;           /* share of nshards (0 or 1: the whole build); the
                              class quartets are split by jk_shard_plan on
                              their cost, and the partial J/K of the ranks
                              sum to the full J/K (all-reduce them)            */
    int reserved[6];
} jk_opts_t;

/*
 * Basis setup for one geometry: device copies of the basis, the Schwarz
 * matrix q[i,j] = sqrt(max |(ij|ij)|) computed on the device, Schwarz-sorted
 * shell-pair lists per lower-triangular group pair (kept if q > cutoff; the
 * upper triangle of diagonal blocks dropped unless diag_block_with_triu),
 * and the primitive-pair cache.
 * Replaces GINTinit_basis_prod_cpu (cuobc/lib/gint/nr_fill_ao_ints.cu:452-470),
 * GINTinit_basis_prod_gpu (nr_fill_ao_ints.cu:472-491) and the q_cond /
 * pair-list part of _VHFOpt.build (cuobc/scf/hf.py:341-408).  Unlike the
 * reference it copies every input, so nothing is borrowed from the caller.
 * atm/bas/env: libcint arrays of the working basis; group_offsets: ngroups+1
 * shell offsets of the (l, nprim) groups (l_ctr_offsets).
 */
int jk_basis_create(const int *atm, int natm, const int *bas, int nbas, const double *env, int nenv,
                    const int *group_offsets, int ngroups, double cutoff, int diag_block_with_triu,
                    jk_basis_t **out);

/* Replaces GINTdel_basis_prod (cuobc/lib/gint/nr_fill_ao_ints.cu:394-410). */
int jk_basis_destroy(jk_basis_t *basis);

/* info[7] = {nbas, nao, ngroups, nclass_pairs, npairs, nprim_pairs,
 * nclass_quartets}.  Mirrors the BasisProdCache fields the reference reads
 * through ctypes (cuobc/scf/hf.py:451-478). */
int jk_basis_info(const jk_basis_t *basis, int *info);

/* Copies of the pair lists (bas_pair2shls 2 x npairs, bas_pairs_locs
 * ncp+1, log_q npairs) and the Schwarz matrix (nbas x nbas); any output may
 * be NULL.  Same content as _VHFOpt.bas_pair2shls / bas_pairs_locs / log_qs
 * (cuobc/scf/hf.py:391-396). */
int jk_basis_pairs(const jk_basis_t *basis, int *pair2shls, int *pair_locs, double *log_q, double *q_cond);

/*
 * One class pair with host-side log-Schwarz bins, same contract as
 * GINTbuild_jk (cuobc/lib/gvhf/nr_jk_driver.cu:227-284): vj/vk are device
 * buffers (n_dm, nao, nao) accumulated (+=) with element (i, j) at
 * i + nao*j, either may be NULL; dm is the device density in the working
 * basis; bins are host arrays of nbins+1 non-decreasing offsets, nbins <= 64.
 * Asynchronous, as GINTbuild_jk: the bins are passed to the device by value
 * (the host arrays may change once the call returns), the results are there
 * once `stream` reaches them.  The calls of one basis handle share a
 * row-prefix buffer: issue them on one stream (or order their streams).
 */
int jk_build_class_pair(jk_basis_t *basis, double *vj, double *vk, const double *dm, int nao, int n_dm,
                        const int *bins_locs_ij, const int *bins_locs_kl, int nbins, int cp_ij, int cp_kl,
                        void *stream);

/* Host only: the shell quartets a per-class-pair call computes for these
 * bins (row ij of the class pair's n_ij shell pairs, in ij bin s, pairs with
 * the kl pairs below bins_kl[nbins - s], as the reference's bin loop pairs
 * kl bin b with ij bins below nbins - b, nr_jk_driver.cu:252-280; diag != 0:
 * a diagonal class pair of jk_build_class_pair, kl <= ij).  qoff (may be
 * NULL) receives the n_ij + 1 row prefixes, *total the count. */
int jk_class_pair_tasks(const int *bins_ij, const int *bins_kl, int nbins, int n_ij, int diag, long long *qoff,
                        long long *total);

/*
 * ERI tensor of one class pair, same contract as GINTfill_int2e
 * (cuobc/lib/gint/nr_fill_ao_ints.cu:493-549): for every (ij, kl) the host
 * bins keep (kl bin b with ij bins below nbins - b, no triangle restriction
 * on a diagonal class pair; cp_kl may exceed cp_ij), eri[(a - o[0])*s[0] + (b - o[1])*s[1] +
 * (c - o[2])*s[2] + (d - o[3])*s[3]] += (ab|cd) over the Cartesian
 * functions of the four shells; eri is a device buffer, strides s[4] and AO
 * offsets o[4] (working-basis AO indices) host arrays.  Pairs on the
 * diagonal of a shell carry the basis's diagonal factor (1 with
 * diag_block_with_triu, else 1/2), as the reference's pair data do.  Every
 * class up to (ii|ii).  Asynchronous with the bin rules of
 * jk_build_class_pair (nbins <= 64, one stream per basis handle).
 */
int jk_fill_int2e(jk_basis_t *basis, double *eri, int nao, const int *strides, const int *ao_offsets,
                  const int *bins_locs_ij, const int *bins_locs_kl, int nbins, int cp_ij, int cp_kl, void *stream);

/*
 * Same computation and buffer contract as jk_build_class_pair, for callers
 * that must not allocate device memory while they run (a serving process or
 * host framework that owns all GPU memory through its own pool and cannot
 * have a library call cudaMalloc behind it).  No counterpart in the
 * reference.  It allocates nothing: its scratch is a fixed device array of
 * about 1 MB inside libjk.so, held on every GPU that loads the library.
 * Limits: at most 131072 shell pairs in the ij class and nbins <= 1024;
 * larger requests return JK_ERR_ARG.  The bins must be non-decreasing with
 * bins_locs_kl[nbins] <= the kl class's pair count (larger counts are
 * clamped to it).  The first call on a device looks up the array's device
 * address (make it before any stream capture); with CUDA's lazy module
 * loading that lookup is also when the array is placed on the device, so a
 * caller whose pool reserves most of the memory should make one call with
 * vj = vk = NULL (which does only the lookup) before the reservation.  Like
 * jk_build_class_pair it returns after the GPU work has finished.  All calls
 * share the array: calls whose GPU work overlaps race and must be serialised
 * by the caller.
 */
int jk_build_class_pair_noalloc(jk_basis_t *basis, double *vj, double *vk, const double *dm, int nao, int n_dm,
                                const int *bins_locs_ij, const int *bins_locs_kl, int nbins, int cp_ij, int cp_kl,
                                void *stream);

/*
 * All class pairs in one call with the screening done on the device: the
 * per-group density condensation, the class-level density screen and the
 * log-Schwarz bin test per quartet, with the reference's decisions
 * (cuobc/scf/hf.py:104-160).  Same buffer contract as jk_build_class_pair.
 * Replaces the task loop of get_jk (cuobc/scf/hf.py:111-166).
 */
int jk_build(jk_basis_t *basis, const double *dm, int n_dm, double *vj, double *vk, const jk_opts_t *opts,
             void *stream);

/*
 * Split of n weighted tasks over nshards owners (the class quartets of a
 * sharded build, weighted by their unscreened work): longest first, each to
 * the owner with the least work so far (ties: lower index), so every rank
 * computes the same plan.  owner[i] in [0, nshards).  Host code only.  The
 * reference farms class pairs to GPUs dynamically from a Python task loop
 * (cuobc/lib/multigpu.py:136-329, cuobc/scf/hf.py:165-169); a static
 * plan needs no coordination between ranks.
 */
int jk_shard_plan(const double *cost, int n, int nshards, int *owner);

/*
 * Full J/K in the caller's basis: dms = C D C^T, jk_build, then
 * J = 2 C^T (V + V^T) C and K = C^T (V + V^T) C (cuobc/scf/hf.py:67-181).
 * coeff: device (nao, nao0) row-major (the working basis -> caller basis map);
 * dm0, vj0, vk0: device (n_dm, nao0, nao0) row-major; vj0/vk0 are
 * overwritten; either may be NULL.
 */
int jk_get_jk(jk_basis_t *basis, const double *coeff, int nao0, const double *dm0, int n_dm, double *vj0,
              double *vk0, const jk_opts_t *opts, void *stream);

/*
 * Batched builds over many molecules (one jk_basis each, same device).  No
 * single reference counterpart: the reference builds one molecule at a time
 * through the task loop of get_jk (cuobc/scf/hf.py:111-166); a batch runs
 * the class quartets of all molecules that share a class (angular momenta,
 * and primitive counts for the team kernels) as one launch, largest
 * molecules' work first, with the same screening decisions as jk_build for
 * each molecule.  Each launch takes static chunks or runs persistent (a grid
 * of the device's resident capacity taking chunks from a device counter),
 * as jk_batch_tune chose; untuned batches use static chunks.  A class
 * quartet with at least `solo_tasks` unscreened tasks (shell-pair rows x
 * columns) is not merged: it runs as its own single-molecule launch, as
 * jk_build makes it; solo_tasks <= 0 merges everything.  jk_batch_create
 * uses JK_BATCH_SOLO_TASKS.
 */
#define JK_BATCH_SOLO_TASKS (1LL << 14)
int jk_batch_create(jk_basis_t *const *bases, int nmol, jk_batch_t **out);
int jk_batch_create_ex(jk_basis_t *const *bases, int nmol, long long solo_tasks, jk_batch_t **out);
int jk_batch_destroy(jk_batch_t *batch);
/* number of class quartets of the batch launched on their own */
int jk_batch_nsolo(const jk_batch_t *batch, int *nsolo);

/* Per molecule m: dms[m] device density in the working basis, vjs[m]/vks[m]
 * device buffers accumulated as in jk_build (either array may be NULL).  The
 * segment tables follow the pointers: a call with new pointers synchronises
 * `stream` once to rebuild them; with the same pointers the call is fully
 * asynchronous. */
int jk_batch_build(jk_batch_t *batch, const double *const *dms, double *const *vjs, double *const *vks, int n_dm,
                   const jk_opts_t *opts, void *stream);

/* Autotuner of the batch's launch shapes (no reference counterpart: the
 * reference launches a fixed 256-thread shape per class pair and bin,
 * cuobc/lib/gint/gint.h:52).  Times every candidate shape of every class
 * launch of the batch (static chunks; persistent at one resident grid with
 * three grab sizes, and at two with the middle one) with CUDA events on
 * `stream`, after the
 * bookkeeping of a real build with these arguments (same contract as
 * jk_batch_build), and keeps the fastest.  cache_path (may be NULL): a text
 * file of earlier choices per (class, primitive counts, part, log2 task
 * count), read first (those launches are not timed again) and rewritten
 * with all choices.  The timing runs accumulate into vjs/vks, which are
 * zeroed before return; the call synchronises `stream`. */
int jk_batch_tune(jk_batch_t *batch, const double *const *dms, double *const *vjs, double *const *vks, int n_dm,
                  const jk_opts_t *opts, const char *cache_path, void *stream);

/* Launch shapes of the batch: *nkeys set; if out is not NULL, 12 ints per
 * key: class index, primitive counts of bra and ket pairs (-1: any), task
 * bound, then for the FP64 and FP32 parts: grab (0: static), grid multiple,
 * tuned time in microseconds (-1: not tuned), segments. */
int jk_batch_info(const jk_batch_t *batch, int *nkeys, int *out);

/* Full J/K of every molecule in its own basis (the jk_get_jk contract per
 * molecule): coeffs[m] device (nao_m, nao0s[m]); dm0s[m], vj0s[m], vk0s[m]
 * device (n_dm, nao0, nao0); vj0s/vk0s overwritten, either array may be NULL. */
int jk_batch_get_jk(jk_batch_t *batch, const double *const *coeffs, const int *nao0s, const double *const *dm0s,
                    double *const *vj0s, double *const *vk0s, int n_dm, const jk_opts_t *opts, void *stream);

/* Rys nodes s = t^2 and weights of the product tables, evaluated on the
 * host (for checking the tables).  Returns JK_ERR_ARG for n outside 1..11. */
int jk_rys_roots_host(int n, double x, double *s, double *w);

/* The same tables evaluated by a device kernel through the paths the J/K
 * kernels use (mode 0: all roots from the shared-memory copy, 1: one root at
 * a time from it, 2: one root from the global copy, 3: all roots in single
 * precision as the FP32 quartets of the mixed mode use them, 4: one root at a
 * time in single precision; modes 3 and 4 for n <= 3 only; 5: one root at a
 * time with the root count known at run time, from the global copy, as the
 * generic kernels evaluate them; n = 1 is evaluated from the Boys function in
 * every mode; n <= 13).  x, s, w are device arrays (count,
 * count*n, count*n).  For checking the device evaluation. */
int jk_rys_roots_device(int n, const double *x, int count, double *s, double *w, int mode, void *stream);

/* Per class quartet (8 ints each): cp_ij, cp_kl, li, lj, lk, ll, nprim_ij,
 * nprim_kl.  No reference counterpart: introspection for the cost model. */
int jk_basis_cq_info(const jk_basis_t *basis, int *out);

/* Screened contracted-quartet counts of the last jk_build (synchronises
 * `stream`): out[c] the FP64 quartets of class quartet c, out[ncq + c] its
 * FP32 quartets (mixed mode; 0 otherwise).  out has 2*ncq entries.  No
 * reference counterpart. */
int jk_last_counts(const jk_basis_t *basis, long long *out, void *stream);

/* Measured FMA-pipe peak of the current device in TFLOP/s (fp32 = 0: FP64,
 * 1: FP32), from 8 independent FMA chains per thread over the whole GPU.
 * No reference counterpart: the roofline denominator of the J/K kernels. */
int jk_fma_peak(int fp32, double *tflops);

/* One-electron integrals of the SCF glue, host code: which = 0 overlap,
 * 1 kinetic, 2 nuclear attraction; out (nao_cart, nao_cart) row-major over
 * all contractions of all shells.  PySCF's mol.intor supplies these to the
 * reference (outside the reference repository). */
int jk_int1e_cart(int which, const int *atm, int natm, const int *bas, int nbas, const double *env, double *out);

/* Description of the last failure in the calling thread. */
const char *jk_last_error(void);

#ifdef __cplusplus
}
#endif
#endif
