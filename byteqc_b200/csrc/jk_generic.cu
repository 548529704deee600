// Generic J/K kernel for the classes with a shell above f (g, h and i,
// l = 4, 5, 6), with the angular momenta read at run time.  The reference's
// GPU kernels reach h shells (cuobc/lib/gvhf/g2e.cu:32-996, up to 11 Rys
// roots) and hand quartets with an i shell to PySCF on the CPU
// (cuobc/scf/hf.py:185-218); here i shells run on the GPU too (13 roots at
// (ii|ii)).  Basis sets such as cc-pVQZ or def2-QZVP carry g functions,
// cc-pV5Z h and cc-pV6Z i.  These classes are rare, so the kernel aims at
// correctness with bounded resources; its fixed sizes come from the largest
// l it serves, GL = 5 (every class up to (hh|hh), 86 KB of shared memory,
// two CTAs per SM) or GL = 6 (classes with an i shell, 153 KB, one CTA):
//
//   one CTA per contracted quartet; for every primitive quartet and root the
//   three (axis, root) 2D blocks are built in shared memory (threads 0-2),
//   then every thread owns elements of the six J/K blocks of the quartet
//   (J_ij, J_kl, K_ik, K_il, K_jk, K_jl), sums the integrals times the
//   matching density elements over the other two indices into a shared-memory
//   accumulator (no atomics: one owner per element), and the blocks are
//   added to J and K with one atomic per element at the end.
//
// Digestion, index conventions and density orientation are those of the
// templated kernels (cuobc/lib/gvhf/contract_jk.cu:225-316): output element
// (a, b) at a + nao*b, K-side densities read transposed.
#include "jk_launch.cuh"

#define JK_GEN_THREADS 128
#define JK_FILL_CHUNK 4096

// fixed sizes of the generic kernels serving shells up to l = GL
template <int GL>
struct JKGen {
    static constexpr int NF = (GL + 1) * (GL + 2) / 2;              // Cartesian components of one shell
    static constexpr int GS = (GL + 1) * (GL + 1) * (GL + 1) * (GL + 1);  // entries of one 2D block
    static constexpr int NR = 2 * GL + 1;                           // roots of the largest class
    static constexpr int BLK = NF * NF;
    static constexpr int G1 = 2 * GL + 1;                           // VRR range in n and m
    static constexpr int H1 = GL + 1;
    static constexpr int W = G1 * G1 + H1 * H1 * G1 + 2 * G1;       // recursion scratch of one unit
    static constexpr size_t SMEM = (3 * GS + 12 * BLK + 3 * W) * sizeof(double);
    static constexpr size_t FILL_SMEM = (3 * GS + JK_FILL_CHUNK + 3 * W) * sizeof(double);
    static constexpr size_t QC_SMEM = (3 * GS + BLK + 3 * W) * sizeof(double);
    static constexpr int CTAS = GL <= 5 ? 2 : 1;                    // resident CTAs per SM
};
static_assert(JKGen<5>::SMEM <= 227 * 1024 && JKGen<6>::SMEM <= 227 * 1024, "generic kernel shared memory");

// One Rys 2D block at run-time angular momenta: the recursion of rys_2d,
// output I[((i*(lj+1)+j)*(lk+1)+k)*(ll+1)+l].  The intermediate arrays live
// in the caller's shared-memory scratch W (JKGen<GL>::W doubles), not on the
// thread's stack, which would reserve local memory for every resident thread
// of the device.
template <int GL>
__device__ void rys_2d_rt(int li, int lj, int lk, int ll, double seed, double c00, double c0p, double b10,
                          double b01, double b00, double dij, double dkl, double* __restrict__ W,
                          double* __restrict__ I) {
    constexpr int G1 = JKGen<GL>::G1, H1 = JKGen<GL>::H1;
    const int nm = li + lj, mm = lk + ll;
    double* G = W;                // G[n * G1 + m]
    double* H = G + G1 * G1;      // H[(i * H1 + j) * G1 + m]: bra transfer
    double* A = H + H1 * H1 * G1;
    double* B = A + G1;
    G[0] = seed;
    for (int n = 0; n < nm; n++) G[(n + 1) * G1] = c00 * G[n * G1] + (n ? n * b10 * G[(n - 1) * G1] : 0.);
    for (int m = 0; m < mm; m++)
        for (int n = 0; n <= nm; n++) {
            double v = c0p * G[n * G1 + m];
            if (m) v += m * b01 * G[n * G1 + m - 1];
            if (n) v += n * b00 * G[(n - 1) * G1 + m];
            G[n * G1 + m + 1] = v;
        }
    const int SK = ll + 1, SJ = (lk + 1) * SK, SI = (lj + 1) * SJ;
    for (int m = 0; m <= mm; m++) {
        for (int a = 0; a <= nm; a++) A[a] = G[a * G1 + m];
        for (int i = 0; i <= li; i++) H[(i * H1) * G1 + m] = A[i];
        for (int j = 1; j <= lj; j++) {
            for (int a = 0; a + j <= nm; a++) A[a] = A[a + 1] + dij * A[a];
            for (int i = 0; i <= li; i++) H[(i * H1 + j) * G1 + m] = A[i];
        }
    }
    for (int i = 0; i <= li; i++)  // ket transfer
        for (int j = 0; j <= lj; j++) {
            for (int c = 0; c <= mm; c++) B[c] = H[(i * H1 + j) * G1 + c];
            for (int k = 0; k <= lk; k++) I[i * SI + j * SJ + k * SK] = B[k];
            for (int l = 1; l <= ll; l++) {
                for (int c = 0; c + l <= mm; c++) B[c] = B[c + 1] + dkl * B[c];
                for (int k = 0; k <= lk; k++) I[i * SI + j * SJ + k * SK + l] = B[k];
            }
        }
}

// the (axis d, root) block of a primitive quartet (jk_unit at run-time l)
template <int GL>
__device__ void jk_unit_rt(const JKPrim& p, double s, double w, int d, double norm, const double* ri,
                           const double* rj, const double* rk, const double* rl, int li, int lj, int lk, int ll,
                           double* W, double* out) {
    const double siAB = s * p.iAB;
    const double bs = p.B * siAB, as = p.A * siAB;
    const double b00 = 0.5 * siAB;
    const double b10 = 0.5 * p.iA * (1. - bs);
    const double b01 = 0.5 * p.iB * (1. - as);
    const double pq = p.P[d] - p.Q[d];
    const double c00 = (p.P[d] - ri[d]) - bs * pq;
    const double c0p = (p.Q[d] - rk[d]) + as * pq;
    const double seed = d == 0 ? norm : (d == 1 ? p.sy : w);
    rys_2d_rt<GL>(li, lj, lk, ll, seed, c00, c0p, b10, b01, b00, ri[d] - rj[d], rk[d] - rl[d], W, out);
}

// Cartesian exponents of the components of shell l into ex[c][3]
__device__ void jk_cart_table(int l, int (*ex)[3]) {
    for (int c = threadIdx.x; c < ncart(l); c += blockDim.x) {
        ex[c][0] = cart_lx(l, c);
        ex[c][1] = cart_ly(l, c);
        ex[c][2] = cart_lz(l, c);
    }
}

// ---------------------------------------------------------------------------
// J/K of one class (one segment or a segment table), one quartet per CTA at
// a time; each CTA takes a contiguous chunk of the tasks
// ---------------------------------------------------------------------------
template <int GL, class Src>
__device__ void jk_generic_body(const Src& src) {
    using G = JKGen<GL>;
    extern __shared__ __align__(16) double gsm[];
    double* gI = gsm;                  // 3 x G::GS: the blocks of one root
    double* Dsm = gI + 3 * G::GS;      // density blocks
    double* acc = Dsm + 6 * G::BLK;    // accumulator blocks
    double* wk = acc + 6 * G::BLK;     // 3 x G::W: recursion scratch of threads 0-2
    __shared__ JKQuartet s_q;
    __shared__ const JKSeg* s_sg;
    __shared__ double s_c[12];
    __shared__ JKPrim s_p;
    __shared__ double s_rs[G::NR], s_rw[G::NR];
    __shared__ int s_ex[4][G::NF][3];  // Cartesian exponents of the four shells
    const int tid = threadIdx.x;
    const long long total = src.total();
    unsigned long long* queue = src.queue();
    const long long chunk = queue ? (long long)src.grab() : (total + gridDim.x - 1) / gridDim.x;
    __shared__ long long s_grab;
    long long tbeg = (long long)blockIdx.x * chunk;
    for (;;) {
    if (queue) {  // persistent mode: the block takes `chunk` tasks per round
        __syncthreads();
        if (tid == 0) s_grab = (long long)atomicAdd(queue, (unsigned long long)chunk);
        __syncthreads();
        tbeg = s_grab;
    }
    if (tbeg >= total) break;
    const long long tend = min(total, tbeg + chunk);
    typename Src::Cursor cur;
    if (tid == 0 && tbeg < tend) cur.init(src, tbeg);
    for (long long t = tbeg; t < tend; t++) {
        if (tid == 0) {
            int row, col;
            s_sg = &cur.seek(src, t, row, col);
            s_q = jk_quartet_at(*s_sg, row, col);
            load_pair_centres(*s_sg, s_q.bij, s_c, s_c + 3);
            load_pair_centres(*s_sg, s_q.bkl, s_c + 6, s_c + 9);
        }
        __syncthreads();
        const JKSeg& sg = *s_sg;
        const JKQuartet q = s_q;
        const int li = sg.ls[0], lj = sg.ls[1], lk = sg.ls[2], ll = sg.ls[3];
        const int nfi = ncart(li), nfj = ncart(lj), nfk = ncart(lk), nfl = ncart(ll);
        const int nr = (li + lj + lk + ll) / 2 + 1;
        const int SK = ll + 1, SJ = (lk + 1) * SK, SI = (lj + 1) * SJ;
        for (int sh = 0; sh < 4; sh++) jk_cart_table(sg.ls[sh], s_ex[sh]);
        // accumulator blocks: [0, o1) J_ij, [o1, o2) J_kl, [o2, o3) K_ik,
        // [o3, o4) K_il, [o4, o5) K_jk, [o5, E) K_jl
        const int o1 = nfi * nfj, o2 = o1 + nfk * nfl, o3 = o2 + nfi * nfk, o4 = o3 + nfi * nfl,
                  o5 = o4 + nfj * nfk, E = o5 + nfj * nfl;
        // density blocks, each at the position of the accumulator it feeds:
        // D_kl at 0, D_ij at d1, D_jl at d2, D_jk at d3, D_il at d4, D_ik at d5
        const int d1 = nfk * nfl, d2 = d1 + nfi * nfj, d3 = d2 + nfj * nfl, d4 = d3 + nfj * nfk,
                  d5 = d4 + nfi * nfl;
        const int nao = sg.nao;
        const int npij = sg.pnp ? __ldg(sg.pnp + q.bij) : sg.nprim_ij;
        const int npkl = sg.pnp ? __ldg(sg.pnp + q.bkl) : sg.nprim_kl;
        for (int idm = 0; idm < sg.n_dm; idm++) {
            const double* D = sg.dm + (size_t)idm * nao * nao;
            // densities in the orientation of the templated kernels: J side
            // D[x + nao y], K side transposed, D[y + nao x]
            for (int e = tid; e < E; e += JK_GEN_THREADS) {
                int r, x0, y0, ny;
                bool tr = true;
                if (e < d1) { x0 = q.k0; y0 = q.l0; ny = nfl; r = e; tr = false; }
                else if (e < d2) { x0 = q.i0; y0 = q.j0; ny = nfj; r = e - d1; tr = false; }
                else if (e < d3) { x0 = q.j0; y0 = q.l0; ny = nfl; r = e - d2; }
                else if (e < d4) { x0 = q.j0; y0 = q.k0; ny = nfk; r = e - d3; }
                else if (e < d5) { x0 = q.i0; y0 = q.l0; ny = nfl; r = e - d4; }
                else { x0 = q.i0; y0 = q.k0; ny = nfk; r = e - d5; }
                const int a = r / ny, b = r - a * ny;
                Dsm[e] = tr ? __ldg(D + (y0 + b) + (size_t)nao * (x0 + a))
                            : __ldg(D + (x0 + a) + (size_t)nao * (y0 + b));
                acc[e] = 0.;
            }
            __syncthreads();
            for (int kp = 0; kp < npkl; kp++)
                for (int ip = 0; ip < npij; ip++) {
                    if (tid == 0) s_p = jk_prim2(jk_pp(sg, q.prim_ij + ip * sg.pst_ij), jk_pp(sg, q.prim_kl + kp * sg.pst_kl));
                    __syncthreads();
                    if (tid < nr) rys_root_rt(sg.rys, nr, s_p.x, tid, s_rs[tid], s_rw[tid]);
                    __syncthreads();
                    for (int r = 0; r < nr; r++) {
                        if (tid < 3)
                            jk_unit_rt<GL>(s_p, s_rs[r], s_rw[r], tid, q.norm, s_c, s_c + 3, s_c + 6, s_c + 9, li,
                                           lj, lk, ll, wk + tid * G::W, gI + tid * G::GS);
                        __syncthreads();
                        const double* gx = gI;
                        const double* gy = gI + G::GS;
                        const double* gz = gI + 2 * G::GS;
#define JK_GEN_I(i, j, k, l)                                                                                  \
    (gx[s_ex[0][i][0] * SI + s_ex[1][j][0] * SJ + s_ex[2][k][0] * SK + s_ex[3][l][0]] *                       \
     gy[s_ex[0][i][1] * SI + s_ex[1][j][1] * SJ + s_ex[2][k][1] * SK + s_ex[3][l][1]] *                       \
     gz[s_ex[0][i][2] * SI + s_ex[1][j][2] * SJ + s_ex[2][k][2] * SK + s_ex[3][l][2]])
                        for (int e = tid; e < E; e += JK_GEN_THREADS) {
                            double v = 0.;
                            if (e < o1) {  // J_ij += (ij|kl) D_kl
                                const int i = e / nfj, j = e - i * nfj;
                                for (int k = 0; k < nfk; k++)
                                    for (int l = 0; l < nfl; l++) v += JK_GEN_I(i, j, k, l) * Dsm[k * nfl + l];
                            } else if (e < o2) {  // J_kl += (ij|kl) D_ij
                                const int x = e - o1, k = x / nfl, l = x - k * nfl;
                                for (int i = 0; i < nfi; i++)
                                    for (int j = 0; j < nfj; j++) v += JK_GEN_I(i, j, k, l) * Dsm[d1 + i * nfj + j];
                            } else if (e < o3) {  // K_ik += (ij|kl) D_jl
                                const int x = e - o2, i = x / nfk, k = x - i * nfk;
                                for (int j = 0; j < nfj; j++)
                                    for (int l = 0; l < nfl; l++) v += JK_GEN_I(i, j, k, l) * Dsm[d2 + j * nfl + l];
                            } else if (e < o4) {  // K_il += (ij|kl) D_jk
                                const int x = e - o3, i = x / nfl, l = x - i * nfl;
                                for (int j = 0; j < nfj; j++)
                                    for (int k = 0; k < nfk; k++) v += JK_GEN_I(i, j, k, l) * Dsm[d3 + j * nfk + k];
                            } else if (e < o5) {  // K_jk += (ij|kl) D_il
                                const int x = e - o4, j = x / nfk, k = x - j * nfk;
                                for (int i = 0; i < nfi; i++)
                                    for (int l = 0; l < nfl; l++) v += JK_GEN_I(i, j, k, l) * Dsm[d4 + i * nfl + l];
                            } else {  // K_jl += (ij|kl) D_ik
                                const int x = e - o5, j = x / nfl, l = x - j * nfl;
                                for (int i = 0; i < nfi; i++)
                                    for (int k = 0; k < nfk; k++) v += JK_GEN_I(i, j, k, l) * Dsm[d5 + i * nfk + k];
                            }
                            acc[e] += v;
                        }
#undef JK_GEN_I
                        __syncthreads();  // the next root rebuilds the blocks
                    }
                }
            // add the blocks to J and K
            for (int e = tid; e < E; e += JK_GEN_THREADS) {
                double* V;
                int r, x0, y0, ny;
                if (e < o1) { V = sg.vj; x0 = q.i0; y0 = q.j0; ny = nfj; r = e; }
                else if (e < o2) { V = sg.vj; x0 = q.k0; y0 = q.l0; ny = nfl; r = e - o1; }
                else if (e < o3) { V = sg.vk; x0 = q.i0; y0 = q.k0; ny = nfk; r = e - o2; }
                else if (e < o4) { V = sg.vk; x0 = q.i0; y0 = q.l0; ny = nfl; r = e - o3; }
                else if (e < o5) { V = sg.vk; x0 = q.j0; y0 = q.k0; ny = nfk; r = e - o4; }
                else { V = sg.vk; x0 = q.j0; y0 = q.l0; ny = nfl; r = e - o5; }
                if (!V) continue;
                const int a = r / ny, b = r - a * ny;
                atomicAdd(V + (size_t)idm * nao * nao + (x0 + a) + (size_t)nao * (y0 + b), acc[e]);
            }
            __syncthreads();  // the shared buffers are reused by the next density / quartet
        }
    }
    if (!queue) break;
    }
}

template <int GL>
__global__ void __launch_bounds__(JK_GEN_THREADS) jk_generic_kernel(const __grid_constant__ JKSeg sg,
                                                                    const long long* __restrict__ task0) {
    JKOneSeg src{sg, task0};
    jk_generic_body<GL>(src);
}

template <int GL>
__global__ void __launch_bounds__(JK_GEN_THREADS) jk_generic_kernel_batch(const JKSeg* __restrict__ segs,
                                                                          const long long* __restrict__ segt,
                                                                          int nseg, unsigned long long* queue,
                                                                          int grab) {
    JKSegTable src{segs, segt, nseg, queue, grab};
    jk_generic_body<GL>(src);
}

template <int GL>
static int jk_generic_blocks(long long max_tasks, int nsm) {
    const long long cap = (long long)nsm * JKGen<GL>::CTAS;
    return (int)(max_tasks < cap ? max_tasks : cap);
}

template <int GL>
static cudaError_t jk_launch_generic(const JKSeg& seg, const long long* task0, long long max_tasks, int nsm,
                                     cudaStream_t st) {
    if (max_tasks <= 0) return cudaSuccess;
    static std::atomic<unsigned long long> attr_done{0};
    if (cudaError_t e = jk_smem_attr(jk_generic_kernel<GL>, JKGen<GL>::SMEM, attr_done); e != cudaSuccess) return e;
    jk_generic_kernel<GL><<<jk_generic_blocks<GL>(max_tasks, nsm), JK_GEN_THREADS, JKGen<GL>::SMEM, st>>>(seg,
                                                                                                         task0);
    return cudaGetLastError();
}

template <int GL>
static cudaError_t jk_launch_generic_batch(const JKSeg* segs, const long long* segt, int nseg, long long max_tasks,
                                           int nsm, const JKBatchCfg& cfg, cudaStream_t st) {
    if (max_tasks <= 0 || nseg <= 0) return cudaSuccess;
    static std::atomic<unsigned long long> attr_done{0};
    if (cudaError_t e = jk_smem_attr(jk_generic_kernel_batch<GL>, JKGen<GL>::SMEM, attr_done); e != cudaSuccess)
        return e;
    const int blocks = cfg.queue ? nsm * JKGen<GL>::CTAS * cfg.grid_mul : jk_generic_blocks<GL>(max_tasks, nsm);
    jk_generic_kernel_batch<GL><<<blocks, JK_GEN_THREADS, JKGen<GL>::SMEM, st>>>(segs, segt, nseg, cfg.queue,
                                                                                cfg.grab);
    return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// ERI tensor fill (the reference's GINTfill_int2e, gint/nr_fill_ao_ints.cu:
// 493-549, kernels gint/g2e.cu:1160-1605): for every screened quartet of a
// class pair, eri[(a-o0)*s0 + (b-o1)*s1 + (c-o2)*s2 + (d-o3)*s3] += (ab|cd)
// over the Cartesian components a, b, c, d of the four shells (AO indices of
// the working basis).  Every class up to (hh|hh); one CTA per quartet; the
// quartet's integrals are summed over primitives and roots in a shared-memory
// chunk of up to JK_FILL_CHUNK elements (classes with more components run
// the primitive loop once per chunk), then added to the tensor (classes
// with an i shell use the GL = 6 sizes).  The
// integrals carry no 1/2 on the ij == kl diagonal (that factor belongs to
// the J/K digestion); pairs on the diagonal of a shell carry the basis
// handle's diagonal factor, as the reference's pair data do.
// ---------------------------------------------------------------------------
template <int GL>
__global__ void __launch_bounds__(JK_GEN_THREADS) jk_fill_kernel(const __grid_constant__ JKSeg sg,
                                                                 const long long* __restrict__ task0,
                                                                 const JKFillOut out) {
    using G = JKGen<GL>;
    extern __shared__ __align__(16) double gsm[];
    double* gI = gsm;                     // 3 x G::GS: the blocks of one root
    double* acc = gI + 3 * G::GS;         // JK_FILL_CHUNK integrals of the quartet
    double* wk = acc + JK_FILL_CHUNK;     // 3 x G::W: recursion scratch of threads 0-2
    __shared__ JKQuartet s_q;
    __shared__ double s_c[12];
    __shared__ JKPrim s_p;
    __shared__ double s_rs[G::NR], s_rw[G::NR];
    __shared__ int s_ex[4][G::NF][3];
    const int tid = threadIdx.x;
    const long long total = task0[1];
    const long long chunk = (total + gridDim.x - 1) / gridDim.x;
    const long long tbeg = (long long)blockIdx.x * chunk;
    const long long tend = min(total, tbeg + chunk);
    if (tbeg >= tend) return;
    const int li = sg.ls[0], lj = sg.ls[1], lk = sg.ls[2], ll = sg.ls[3];
    const int nfi = ncart(li), nfj = ncart(lj), nfk = ncart(lk), nfl = ncart(ll);
    const int nf = nfi * nfj * nfk * nfl;
    const int nr = (li + lj + lk + ll) / 2 + 1;
    const int SK = ll + 1, SJ = (lk + 1) * SK, SI = (lj + 1) * SJ;
    for (int sh = 0; sh < 4; sh++) jk_cart_table(sg.ls[sh], s_ex[sh]);
    JKTaskCursor cur;
    if (tid == 0) cur.init(sg, tbeg);
    for (long long t = tbeg; t < tend; t++) {
        if (tid == 0) {
            const int col = cur.seek(sg, t);
            s_q = jk_quartet_at(sg, cur.row, col);
            load_pair_centres(sg, s_q.bij, s_c, s_c + 3);
            load_pair_centres(sg, s_q.bkl, s_c + 6, s_c + 9);
        }
        __syncthreads();
        const JKQuartet q = s_q;
        const int npij = sg.pnp ? __ldg(sg.pnp + q.bij) : sg.nprim_ij;
        const int npkl = sg.pnp ? __ldg(sg.pnp + q.bkl) : sg.nprim_kl;
        for (int c0 = 0; c0 < nf; c0 += JK_FILL_CHUNK) {
            const int c1 = min(nf, c0 + JK_FILL_CHUNK);
            for (int e = c0 + tid; e < c1; e += JK_GEN_THREADS) acc[e - c0] = 0.;
            for (int kp = 0; kp < npkl; kp++)
                for (int ip = 0; ip < npij; ip++) {
                    if (tid == 0)
                        s_p = jk_prim2(jk_pp(sg, q.prim_ij + ip * sg.pst_ij), jk_pp(sg, q.prim_kl + kp * sg.pst_kl));
                    __syncthreads();
                    if (tid < nr) rys_root_rt(sg.rys, nr, s_p.x, tid, s_rs[tid], s_rw[tid]);
                    __syncthreads();
                    for (int r = 0; r < nr; r++) {
                        if (tid < 3)
                            jk_unit_rt<GL>(s_p, s_rs[r], s_rw[r], tid, JK_FAC, s_c, s_c + 3, s_c + 6, s_c + 9, li,
                                           lj, lk, ll, wk + tid * G::W, gI + tid * G::GS);
                        __syncthreads();
                        for (int e = c0 + tid; e < c1; e += JK_GEN_THREADS) {
                            int x = e;
                            const int l = x % nfl;
                            x /= nfl;
                            const int k = x % nfk;
                            x /= nfk;
                            const int j = x % nfj;
                            const int i = x / nfj;
                            double v = 1.;
                            for (int d = 0; d < 3; d++)
                                v *= gI[d * G::GS + s_ex[0][i][d] * SI + s_ex[1][j][d] * SJ + s_ex[2][k][d] * SK +
                                        s_ex[3][l][d]];
                            acc[e - c0] += v;
                        }
                        __syncthreads();  // the next root rebuilds the blocks
                    }
                }
            for (int e = c0 + tid; e < c1; e += JK_GEN_THREADS) {
                int x = e;
                const int l = x % nfl;
                x /= nfl;
                const int k = x % nfk;
                x /= nfk;
                const int j = x % nfj;
                const int i = x / nfj;
                const long long o = (long long)(q.i0 + i - out.off[0]) * out.st[0] +
                                    (long long)(q.j0 + j - out.off[1]) * out.st[1] +
                                    (long long)(q.k0 + k - out.off[2]) * out.st[2] +
                                    (long long)(q.l0 + l - out.off[3]) * out.st[3];
                atomicAdd(out.eri + o, acc[e - c0]);
            }
            __syncthreads();  // acc is reused by the next chunk / quartet
        }
    }
}

template <int GL>
static cudaError_t jk_launch_fill_gl(const JKSeg& seg, const long long* task0, long long max_tasks, int nsm,
                                     const JKFillOut& out, cudaStream_t st) {
    static std::atomic<unsigned long long> attr_done{0};
    if (cudaError_t e = jk_smem_attr(jk_fill_kernel<GL>, JKGen<GL>::FILL_SMEM, attr_done); e != cudaSuccess)
        return e;
    const long long cap = (long long)nsm * 2;  // two CTAs per SM (77 KB at GL = 5, 110 KB at GL = 6)
    const int blocks = (int)(max_tasks < cap ? max_tasks : cap);
    jk_fill_kernel<GL><<<blocks, JK_GEN_THREADS, JKGen<GL>::FILL_SMEM, st>>>(seg, task0, out);
    return cudaGetLastError();
}

jk_fill_fn jk_internal_fill_launcher(int class_idx);

// classes up to f with a templated kernel use it (the thread or team shape
// of their J/K kernel, writing the quartet's block instead of digesting
// it); the others the generic kernel above
cudaError_t jk_launch_fill(const JKSeg& seg, const long long* task0, long long max_tasks, int nsm, double* eri,
                           const long long* strides, const int* offsets, cudaStream_t st) {
    if (max_tasks <= 0) return cudaSuccess;
    JKFillOut out;
    out.eri = eri;
    for (int a = 0; a < 4; a++) {
        out.st[a] = strides[a];
        out.off[a] = offsets[a];
    }
    const int lmax = max(max(seg.ls[0], seg.ls[1]), max(seg.ls[2], seg.ls[3]));
    if (lmax <= JK_LMAX) {
        jk_fill_fn f = jk_internal_fill_launcher(JK_CLASS_INDEX(seg.ls[0], seg.ls[1], seg.ls[2], seg.ls[3]));
        if (f) return f(seg, task0, max_tasks, nsm, out, st);
    }
    return lmax <= 5 ? jk_launch_fill_gl<5>(seg, task0, max_tasks, nsm, out, st)
                     : jk_launch_fill_gl<6>(seg, task0, max_tasks, nsm, out, st);
}

// every class with a shell above f runs the generic kernel, in FP64 also for
// the FP32 part of the mixed mode
void jk_register_generic(JKTables* T) {
    for (int li = 0; li <= JK_LMAX_ALL; li++)
        for (int lj = 0; lj <= li; lj++)
            for (int lk = 0; lk <= JK_LMAX_ALL; lk++)
                for (int ll = 0; ll <= lk; ll++) {
                    if (li <= JK_LMAX && lk <= JK_LMAX) continue;
                    const int c = JK_CLASS_INDEX(li, lj, lk, ll);
                    const bool six = li == 6 || lk == 6;  // li >= lj, lk >= ll
                    T->t64[c] = T->t32[c] = six ? jk_launch_generic<6> : jk_launch_generic<5>;
                    T->b64[c] = T->b32[c] = six ? jk_launch_generic_batch<6> : jk_launch_generic_batch<5>;
                }
}

// ---------------------------------------------------------------------------
// Schwarz diagonal q = sqrt(max |(ab|ab)|) of the pairs with a shell above f
// (the quantity jk_qcond_kernel gives the lower classes): one CTA per pair,
// the diagonal elements owned by the threads
// ---------------------------------------------------------------------------
template <int GL>
__global__ void __launch_bounds__(JK_GEN_THREADS) jk_qcond_generic_kernel(
    const int* __restrict__ pi, const int* __restrict__ pj, int npairs, const int* __restrict__ atm,
    const int* __restrict__ bas, const double* __restrict__ env, int nbas, double* __restrict__ q,
    const double* __restrict__ rys) {
    using G = JKGen<GL>;
    extern __shared__ __align__(16) double gsm[];
    double* gI = gsm;
    double* diag = gI + 3 * G::GS;
    double* wk = diag + G::BLK;
    __shared__ JKPrim s_p;
    __shared__ double s_rs[G::NR], s_rw[G::NR], s_c[6];
    __shared__ int s_ex[2][G::NF][3];
    __shared__ double s_red[JK_GEN_THREADS];
    const int tid = threadIdx.x;
    for (int p = blockIdx.x; p < npairs; p += gridDim.x) {
        const int ish = pi[p], jsh = pj[p];
        const int li = bas[ish * BAS_SLOTS + ANG_OF], lj = bas[jsh * BAS_SLOTS + ANG_OF];
        const int nfi = ncart(li), nfj = ncart(lj);
        const int nr = li + lj + 1;  // (li lj | li lj)
        const int SK = lj + 1, SJ = (li + 1) * SK, SI = (lj + 1) * SJ;
        const double* ri = env + atm[bas[ish * BAS_SLOTS + ATOM_OF] * ATM_SLOTS + PTR_COORD];
        const double* rj = env + atm[bas[jsh * BAS_SLOTS + ATOM_OF] * ATM_SLOTS + PTR_COORD];
        const int npi = bas[ish * BAS_SLOTS + NPRIM_OF], npj = bas[jsh * BAS_SLOTS + NPRIM_OF];
        const double* ai = env + bas[ish * BAS_SLOTS + PTR_EXP];
        const double* aj = env + bas[jsh * BAS_SLOTS + PTR_EXP];
        const double* ci = env + bas[ish * BAS_SLOTS + PTR_COEFF];
        const double* cj = env + bas[jsh * BAS_SLOTS + PTR_COEFF];
        const double fsp = (li == 0 ? 0.282094791773878143 : (li == 1 ? 0.488602511902919921 : 1.0)) *
                           (lj == 0 ? 0.282094791773878143 : (lj == 1 ? 0.488602511902919921 : 1.0));
        if (tid < 3) {
            s_c[tid] = ri[tid];
            s_c[3 + tid] = rj[tid];
        }
        jk_cart_table(li, s_ex[0]);
        jk_cart_table(lj, s_ex[1]);
        for (int e = tid; e < nfi * nfj; e += JK_GEN_THREADS) diag[e] = 0.;
        double r2 = 0;
        for (int d = 0; d < 3; d++) r2 += (ri[d] - rj[d]) * (ri[d] - rj[d]);
        __syncthreads();
        for (int ip = 0; ip < npi; ip++)
            for (int jp = 0; jp < npj; jp++)
                for (int kp = 0; kp < npi; kp++)
                    for (int lp = 0; lp < npj; lp++) {
                        if (tid == 0) {
                            const double A = ai[ip] + aj[jp], B = ai[kp] + aj[lp];
                            const double eij = fsp * ci[ip] * cj[jp] * exp(-r2 * ai[ip] * aj[jp] / A);
                            const double ekl = fsp * ci[kp] * cj[lp] * exp(-r2 * ai[kp] * aj[lp] / B);
                            JKPrim pr;
                            pr.A = A;
                            pr.B = B;
                            pr.AB = A + B;
                            pr.iA = 1. / A;
                            pr.iB = 1. / B;
                            pr.iAB = 1. / pr.AB;
                            for (int d = 0; d < 3; d++) {
                                pr.P[d] = (ai[ip] * ri[d] + aj[jp] * rj[d]) / A;
                                pr.Q[d] = (ai[kp] * ri[d] + aj[lp] * rj[d]) / B;
                            }
                            const double dx = pr.P[0] - pr.Q[0], dy = pr.P[1] - pr.Q[1], dz = pr.P[2] - pr.Q[2];
                            pr.x = A * B / pr.AB * (dx * dx + dy * dy + dz * dz);
                            pr.sy = eij * ekl / (sqrt(pr.AB) * A * B);
                            s_p = pr;
                        }
                        __syncthreads();
                        if (tid < nr) rys_root_rt(rys, nr, s_p.x, tid, s_rs[tid], s_rw[tid]);
                        __syncthreads();
                        for (int r = 0; r < nr; r++) {
                            if (tid < 3)
                                jk_unit_rt<GL>(s_p, s_rs[r], s_rw[r], tid, JK_FAC, s_c, s_c + 3, s_c, s_c + 3, li,
                                               lj, li, lj, wk + tid * G::W, gI + tid * G::GS);
                            __syncthreads();
                            for (int e = tid; e < nfi * nfj; e += JK_GEN_THREADS) {
                                const int a = e / nfj, b = e - a * nfj;
                                double v = 1.;
                                for (int d = 0; d < 3; d++)
                                    v *= gI[d * G::GS + s_ex[0][a][d] * (SI + SK) + s_ex[1][b][d] * (SJ + 1)];
                                diag[e] += v;
                            }
                            __syncthreads();
                        }
                    }
        double mx = 0.;
        for (int e = tid; e < nfi * nfj; e += JK_GEN_THREADS) mx = fmax(mx, fabs(diag[e]));
        s_red[tid] = mx;
        __syncthreads();
        for (int o = JK_GEN_THREADS / 2; o > 0; o >>= 1) {
            if (tid < o) s_red[tid] = fmax(s_red[tid], s_red[tid + o]);
            __syncthreads();
        }
        if (tid == 0) {
            const double v = sqrt(s_red[0]);
            q[(size_t)ish * nbas + jsh] = v;
            q[(size_t)jsh * nbas + ish] = v;
        }
        __syncthreads();
    }
}

template <int GL>
static void jk_qcond_generic_gl(const int* pi, const int* pj, int n, const int* atm, const int* bas,
                                const double* env, int nbas, double* q, const double* rys, cudaStream_t st) {
    static std::atomic<unsigned long long> attr_done{0};
    // a failure here shows up in the caller's cudaGetLastError
    if (jk_smem_attr(jk_qcond_generic_kernel<GL>, JKGen<GL>::QC_SMEM, attr_done) != cudaSuccess) return;
    const int blocks = n < 4096 ? n : 4096;
    jk_qcond_generic_kernel<GL><<<blocks, JK_GEN_THREADS, JKGen<GL>::QC_SMEM, st>>>(pi, pj, n, atm, bas, env, nbas,
                                                                                   q, rys);
}

// lmax: the larger angular momentum of the pairs in the list (4..6)
void jk_qcond_generic(const int* pi, const int* pj, int n, const int* atm, const int* bas, const double* env,
                      int nbas, double* q, const double* rys, int lmax, cudaStream_t st) {
    if (n <= 0) return;
    if (lmax <= 5)
        jk_qcond_generic_gl<5>(pi, pj, n, atm, bas, env, nbas, q, rys, st);
    else
        jk_qcond_generic_gl<6>(pi, pj, n, atm, bas, env, nbas, q, rys, st);
}
