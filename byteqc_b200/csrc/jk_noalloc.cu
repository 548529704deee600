// jk_build_class_pair_noalloc: the per-class-pair J/K build with its scratch
// memory in a fixed device array instead of buffers the library allocates.
//
// Who needs it: callers that must not allocate device memory once they are
// running.  A serving process or a host framework that reserves the GPU's
// memory up front through its own pool cannot let a library call cudaMalloc
// behind its back (the allocation can fail against the pool's reservation,
// fragments memory the pool manages, and cudaMalloc/cudaFree may synchronise
// the device in the middle of latency-critical work).  jk_build_class_pair
// allocates its row-offset and segment buffers on first use and grows them
// when a larger class pair comes; this entry point never does.
//
// How: the scratch (row offsets, task counts and the bins) lives in the
// file-scope array jk_na_scratch below, sized for at most JK_NA_MAX_ROWS
// shell pairs in the ij class and JK_NA_MAX_BINS bins.  Every GPU that loads
// this module holds the array (about 1 MB) until the process exits.  Host
// code cannot use the array's name as a device address (in host code it
// names a host-side stand-in), so the first call on each device looks the
// address up with cudaGetSymbolAddress, with that device current, and caches
// it; that first call should come before any stream capture.  With CUDA's
// lazy module loading (the default) the array is placed on a device only at
// that lookup, so a caller whose pool reserves most of the device's memory
// should make the first call (a call with vj = vk = NULL does only the
// lookup) before the reservation, or run with CUDA_MODULE_LOADING=EAGER.
// The cached address is not valid after cudaDeviceReset.  All calls share
// the one array and the previous call's contents stay in it: every field a
// call reads is rewritten by that call before use.  Calls whose GPU work
// overlaps (on different streams, or from different threads) race on the
// array and must be serialised by the caller.  Like jk_build_class_pair, the
// call returns after its GPU work has finished (it synchronises the stream),
// so the host bins and the outputs are free to use on return.
#include <mutex>

#include "jk_internal.h"

#define JK_NA_MAX_ROWS (1 << 17)  // shell pairs of the ij class
#define JK_NA_MAX_BINS 1024
#define JK_NA_OFF_TASK0 0
#define JK_NA_OFF_BINS 256
#define JK_NA_OFF_QOFF (JK_NA_OFF_BINS + 2 * (JK_NA_MAX_BINS + 1) * 4 + 256)
#define JK_NA_BYTES (JK_NA_OFF_QOFF + (JK_NA_MAX_ROWS + 1) * 8)

static __device__ __align__(256) unsigned char jk_na_scratch[JK_NA_BYTES];

static_assert(JK_NA_OFF_QOFF % 8 == 0, "qoff alignment");

static std::mutex g_na_mu;
static unsigned char* g_na_ptr[64];

// device address of jk_na_scratch on the current device (looked up once)
static int na_scratch(unsigned char** out) {
    int dev;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return jk_internal_set_err(JK_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= 64) return jk_internal_set_err(JK_ERR_ARG, "device ordinal out of range");
    std::lock_guard<std::mutex> lk(g_na_mu);
    if (!g_na_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, jk_na_scratch);
        if (e != cudaSuccess) return jk_internal_set_err(JK_ERR_CUDA, cudaGetErrorString(e));
        g_na_ptr[dev] = (unsigned char*)p;
    }
    *out = g_na_ptr[dev];
    return JK_OK;
}

// Row offsets of one class pair from the reference's host bins
// (cuobc/lib/gvhf/nr_jk_driver.cu:252-280): row ij in bin s keeps
// kl < bins_kl[nbins - s]; a diagonal class pair keeps kl <= ij.
// One block; writes qoff[0..n_ij] and task0 = {0, total}.  A count is
// clamped to the n_kl pairs of the kl class, so bins beyond the class cannot
// take the task total past the launch bound.
__global__ void jk_na_qoff_kernel(const int* __restrict__ bins_ij, const int* __restrict__ bins_kl, int nbins,
                                  int n_ij, int n_kl, int diag, long long* __restrict__ qoff,
                                  long long* __restrict__ task0) {
    __shared__ long long carry;
    __shared__ long long wsum[32];
    if (threadIdx.x == 0) {
        carry = 0;
        qoff[0] = 0;
    }
    __syncthreads();
    for (int base = 0; base < n_ij; base += blockDim.x) {
        int ij = base + threadIdx.x;
        long long cnt = 0;
        if (ij < n_ij && ij >= bins_ij[0] && bins_kl[0] == 0) {
            int lo = 0, hi = nbins;  // smallest s with ij < bins_ij[s + 1]
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (ij < bins_ij[mid + 1]) hi = mid; else lo = mid + 1;
            }
            if (lo < nbins) {
                cnt = bins_kl[nbins - lo];
                if (cnt > n_kl) cnt = n_kl;
                if (cnt < 0) cnt = 0;
                if (diag && cnt > ij + 1) cnt = ij + 1;
            }
        }
        long long v = cnt;
        int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
        for (int o = 1; o < 32; o <<= 1) {
            long long y = __shfl_up_sync(0xffffffffu, v, o);
            if (lane >= o) v += y;
        }
        if (lane == 31) wsum[warp] = v;
        __syncthreads();
        if (warp == 0) {
            long long w = (lane < (int)(blockDim.x >> 5)) ? wsum[lane] : 0;
            for (int o = 1; o < 32; o <<= 1) {
                long long y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            wsum[lane] = w;
        }
        __syncthreads();
        long long incl = v + (warp ? wsum[warp - 1] : 0) + carry;
        if (ij < n_ij) qoff[ij + 1] = incl;
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) carry = incl;
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        task0[0] = 0;
        task0[1] = carry;
    }
}

extern "C" int jk_build_class_pair_noalloc(jk_basis_t* b, double* vj, double* vk, const double* dm, int nao, int n_dm,
                                           const int* bins_locs_ij, const int* bins_locs_kl, int nbins, int cp_ij,
                                           int cp_kl, void* stream) {
    if (!b || !dm || !bins_locs_ij || !bins_locs_kl || nbins <= 0 || n_dm <= 0)
        return jk_internal_set_err(JK_ERR_ARG, "jk_build_class_pair_noalloc: invalid arguments");
    if (nbins > JK_NA_MAX_BINS)
        return jk_internal_set_err(JK_ERR_ARG, "jk_build_class_pair_noalloc: nbins exceeds the 1024 maximum");
    int n_ij, n_kl, nao_b;
    int rc = jk_internal_class_info(b, cp_ij, cp_kl, &n_ij, &n_kl, &nao_b);
    if (rc) return rc;
    if (nao != nao_b) return jk_internal_set_err(JK_ERR_ARG, "jk_build_class_pair_noalloc: nao does not match");
    if (n_ij > JK_NA_MAX_ROWS)
        return jk_internal_set_err(JK_ERR_ARG,
                                   "jk_build_class_pair_noalloc: the ij class has more than 131072 shell pairs; "
                                   "use jk_build_class_pair");
    unsigned char* sc;
    rc = na_scratch(&sc);
    if (rc) return rc;
    if (!vj && !vk) return JK_OK;
    cudaStream_t st = (cudaStream_t)stream;
    long long* d_task0 = (long long*)(sc + JK_NA_OFF_TASK0);
    int* d_bins_ij = (int*)(sc + JK_NA_OFF_BINS);
    int* d_bins_kl = d_bins_ij + (nbins + 1);
    long long* d_qoff = (long long*)(sc + JK_NA_OFF_QOFF);
    cudaError_t e = cudaMemcpyAsync(d_bins_ij, bins_locs_ij, sizeof(int) * (nbins + 1), cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_bins_kl, bins_locs_kl, sizeof(int) * (nbins + 1), cudaMemcpyHostToDevice, st);
    JKSeg seg;
    jk_internal_fill_seg(b, cp_ij, cp_kl, d_qoff, n_ij, dm, n_dm, vj, vk, &seg);
    if (e != cudaSuccess) return jk_internal_set_err(JK_ERR_CUDA, cudaGetErrorString(e));
    jk_na_qoff_kernel<<<1, 1024, 0, st>>>(d_bins_ij, d_bins_kl, nbins, n_ij, n_kl, cp_ij == cp_kl, d_qoff, d_task0);
    e = cudaGetLastError();
    if (e != cudaSuccess) return jk_internal_set_err(JK_ERR_CUDA, cudaGetErrorString(e));
    long long max_tasks = cp_ij == cp_kl ? (long long)n_ij * (n_ij + 1) / 2 : (long long)n_ij * n_kl;
    rc = jk_internal_launch(b, cp_ij, cp_kl, seg, d_task0, max_tasks, stream);
    if (rc) return rc;
    // same synchronous contract as jk_build_class_pair
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return jk_internal_set_err(JK_ERR_CUDA, cudaGetErrorString(e));
    return JK_OK;
}
