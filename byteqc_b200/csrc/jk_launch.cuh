// Launchers of the J/K kernels, one per (li, lj, lk, ll) class and arithmetic
// type, collected in a table indexed by JK_CLASS_INDEX(li, lj, lk, ll).
#pragma once
#include <atomic>

#include "jk_kernels.cuh"

// cudaFuncSetAttribute acts on the current device only, so the "already set"
// flag of a kernel is kept per device (bit d of `done` for device d < 64;
// devices beyond that set the attribute on every launch).
template <class K>
cudaError_t jk_smem_attr(K kernel, size_t smem, std::atomic<unsigned long long>& done) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (bit && (done.load(std::memory_order_relaxed) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && bit) done.fetch_or(bit, std::memory_order_relaxed);
    return e;
}


// One class quartet (one segment): the segment descriptor goes by value into
// the kernel's parameter space; task0[1] (device) holds the task count.
template <int LI, int LJ, int LK, int LL, typename R>
cudaError_t jk_launch(const JKSeg& seg, const long long* task0, long long max_tasks, int nsm, cudaStream_t st) {
    using C = JKClass<LI, LJ, LK, LL>;
    if (max_tasks <= 0) return cudaSuccess;
    if constexpr (C::P == 0) {
        constexpr size_t smem = RysS<C::NROOTS>::WORDS * sizeof(double);
        static std::atomic<unsigned long long> attr_done{0};
        if (cudaError_t e = jk_smem_attr(jk_thread_kernel<C, R>, smem, attr_done); e != cudaSuccess) return e;
        long long want = (max_tasks + 127) / 128;
        long long cap = (long long)nsm * 16;
        int blocks = (int)(want < cap ? want : cap);
        jk_thread_kernel<C, R><<<blocks, 128, smem, st>>>(seg, task0);
    } else {
        using S = JKTeamShape<C>;
        constexpr size_t smem = jk_team_smem<C, R>();
        static std::atomic<unsigned long long> attr_done{0};
        if (cudaError_t e = jk_smem_attr(jk_team_kernel<C, R>, smem, attr_done); e != cudaSuccess) return e;
        long long want = (max_tasks + S::QPB - 1) / S::QPB;
        long long cap = (long long)nsm * 8;
        int blocks = (int)(want < cap ? want : cap);
        jk_team_kernel<C, R><<<blocks, S::THREADS, smem, st>>>(seg, task0);
    }
    return cudaGetLastError();
}

// resident blocks per SM of a kernel at a launch shape, looked up once per
// device (bit d of `done`, the count in cnt[d])
template <class K>
int jk_resident_blocks(K kernel, int threads, size_t smem, std::atomic<unsigned long long>& done, int* cnt) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return 1;
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cnt[dev];
    int nb = 1;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kernel, threads, smem) != cudaSuccess || nb < 1) nb = 1;
    if (bit) {
        cnt[dev] = nb;
        done.fetch_or(bit, std::memory_order_release);
    }
    return nb;
}

// Batched launch: the segments of one class (same angular momenta and
// primitive counts) of many molecules, task prefix segt[0..nseg] on the
// device; static chunks or the persistent mode (JKBatchCfg).
template <int LI, int LJ, int LK, int LL, typename R>
cudaError_t jk_launch_batch(const JKSeg* segs, const long long* segt, int nseg, long long max_tasks, int nsm,
                            const JKBatchCfg& cfg, cudaStream_t st) {
    using C = JKClass<LI, LJ, LK, LL>;
    if (max_tasks <= 0 || nseg <= 0) return cudaSuccess;
    if constexpr (C::P == 0) {
        constexpr size_t smem = RysS<C::NROOTS>::WORDS * sizeof(double);
        static std::atomic<unsigned long long> attr_done{0};
        if (cudaError_t e = jk_smem_attr(jk_thread_kernel_batch<C, R>, smem, attr_done); e != cudaSuccess) return e;
        int blocks;
        if (cfg.queue) {
            static std::atomic<unsigned long long> occ_done{0};
            static int occ[64];
            blocks = nsm * cfg.grid_mul * jk_resident_blocks(jk_thread_kernel_batch<C, R>, 128, smem, occ_done, occ);
        } else {
            long long want = (max_tasks + 127) / 128;
            long long cap = (long long)nsm * 16;
            blocks = (int)(want < cap ? want : cap);
        }
        jk_thread_kernel_batch<C, R><<<blocks, 128, smem, st>>>(segs, segt, nseg, cfg.queue, cfg.grab);
    } else {
        using S = JKTeamShape<C>;
        constexpr size_t smem = jk_team_smem<C, R>();
        static std::atomic<unsigned long long> attr_done{0};
        if (cudaError_t e = jk_smem_attr(jk_team_kernel_batch<C, R>, smem, attr_done); e != cudaSuccess) return e;
        int blocks;
        if (cfg.queue) {
            static std::atomic<unsigned long long> occ_done{0};
            static int occ[64];
            blocks = nsm * cfg.grid_mul *
                     jk_resident_blocks(jk_team_kernel_batch<C, R>, S::THREADS, smem, occ_done, occ);
        } else {
            long long want = (max_tasks + S::QPB - 1) / S::QPB;
            long long cap = (long long)nsm * 8;
            blocks = (int)(want < cap ? want : cap);
        }
        jk_team_kernel_batch<C, R><<<blocks, S::THREADS, smem, st>>>(segs, segt, nseg, cfg.queue, cfg.grab);
    }
    return cudaGetLastError();
}

// ERI-tensor fill of one class quartet with the class's templated kernel
// (thread or team shape, FP64), same grid as the J/K launch
template <int LI, int LJ, int LK, int LL>
cudaError_t jk_launch_fill_t(const JKSeg& seg, const long long* task0, long long max_tasks, int nsm,
                             const JKFillOut& out, cudaStream_t st) {
    using C = JKClass<LI, LJ, LK, LL>;
    if (max_tasks <= 0) return cudaSuccess;
    if constexpr (C::P == 0) {
        constexpr size_t smem = RysS<C::NROOTS>::WORDS * sizeof(double);
        static std::atomic<unsigned long long> attr_done{0};
        if (cudaError_t e = jk_smem_attr(jk_thread_fill_kernel<C>, smem, attr_done); e != cudaSuccess) return e;
        long long want = (max_tasks + 127) / 128;
        long long cap = (long long)nsm * 16;
        int blocks = (int)(want < cap ? want : cap);
        jk_thread_fill_kernel<C><<<blocks, 128, smem, st>>>(seg, task0, out);
    } else {
        using S = JKTeamShape<C>;
        constexpr size_t smem = jk_team_smem<C, double>();
        static std::atomic<unsigned long long> attr_done{0};
        if (cudaError_t e = jk_smem_attr(jk_team_fill_kernel<C>, smem, attr_done); e != cudaSuccess) return e;
        long long want = (max_tasks + S::QPB - 1) / S::QPB;
        long long cap = (long long)nsm * 8;
        int blocks = (int)(want < cap ? want : cap);
        jk_team_fill_kernel<C><<<blocks, S::THREADS, smem, st>>>(seg, task0, out);
    }
    return cudaGetLastError();
}
typedef cudaError_t (*jk_fill_fn)(const JKSeg& seg, const long long* task0, long long max_tasks, int nsm,
                                  const JKFillOut& out, cudaStream_t st);

// launcher tables indexed by JK_CLASS_INDEX(li, lj, lk, ll)
struct JKTables {
    jk_launch_fn t64[JK_NCLASS], t32[JK_NCLASS];
    jk_launch_batch_fn b64[JK_NCLASS], b32[JK_NCLASS];
    // team kernels need one primitive count per launch (their blocks loop
    // over the primitives in step); thread and generic kernels read it per
    // segment
    unsigned char team[JK_NCLASS];
    jk_fill_fn fill[JK_NCLASS];  // templated ERI fill (classes up to f)
};

// classes with a shell above f: the generic kernel (jk_generic.cu)
void jk_register_generic(JKTables* T);

// per-instantiation-file registration (jk_inst_*.cu, generated list)
#include "jk_inst_list.h"

#ifndef JK_NO_FP32
#define JK_REG32(LI, LJ, LK, LL)                                         \
    T->t32[JK_CLASS_INDEX(LI, LJ, LK, LL)] = jk_launch<LI, LJ, LK, LL, float>; \
    T->b32[JK_CLASS_INDEX(LI, LJ, LK, LL)] = jk_launch_batch<LI, LJ, LK, LL, float>;
#else
#define JK_REG32(LI, LJ, LK, LL)
#endif
#define JK_REG(LI, LJ, LK, LL)                                                       \
    T->team[JK_CLASS_INDEX(LI, LJ, LK, LL)] = JKClass<LI, LJ, LK, LL>::P != 0;    \
    T->fill[JK_CLASS_INDEX(LI, LJ, LK, LL)] = jk_launch_fill_t<LI, LJ, LK, LL>;   \
    T->t64[JK_CLASS_INDEX(LI, LJ, LK, LL)] = jk_launch<LI, LJ, LK, LL, double>;  \
    T->b64[JK_CLASS_INDEX(LI, LJ, LK, LL)] = jk_launch_batch<LI, LJ, LK, LL, double>; \
    JK_REG32(LI, LJ, LK, LL)
