// J/K kernels: Rys-quadrature ERIs of contracted shell quartets digested on
// the fly into J and K (the work of the reference's GINTint2e_jk_kernel*,
// cuobc/lib/gvhf/g2e.cu:998-1605, and GINTkernel_getjk,
// cuobc/lib/gvhf/contract_jk.cu:28-635).
//
// Work unit: one screened contracted shell quartet (ij|kl) of one segment.
// All primitive quartets and roots of it are summed in registers before the
// quartet's contribution to J and K is formed, so every J/K element of the
// quartet is written with one atomic, instead of one per primitive and root.
//
// Two execution shapes, fixed per class at compile time (JKClass::P):
//   P = 0  one thread per quartet; the 2D integrals of one root live in
//          registers and all NF Cartesian products accumulate in registers;
//          the digestion goes straight to global atomics;
//   P > 0  a team of T threads per quartet: the 3*NROOTS (axis, root) 2D
//          blocks are built cooperatively in shared memory, each thread owns
//          the leading P Cartesian indices (i, or i and j) and accumulates the
//          remaining components in registers; the digestion reduces the
//          partial J/K blocks of the team in shared memory and flushes each
//          element with one global atomic.
// R is the arithmetic type of the recursion and products (double, or float
// for the mixed-precision path); roots, weights, prefactors and all J/K
// accumulation stay in double.
#pragma once
#include "jk_common.cuh"

__device__ __forceinline__ int jk_find_seg(const long long* __restrict__ task0, int nseg, long long t) {
    int lo = 0, hi = nseg - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (task0[mid] <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

__device__ __forceinline__ int jk_find_row(const long long* __restrict__ qoff, int n, long long t) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        int mid = (lo + hi + 1) >> 1;
        if (__ldg(qoff + mid) <= t) lo = mid; else hi = mid - 1;
    }
    return lo;
}

struct JKQuartet {
    int bij, bkl;          // global pair indices
    int i0, j0, k0, l0;    // first AO of each shell
    int prim_ij, prim_kl;  // first primitive pair of ij and kl (stride sg.pst_ij, sg.pst_kl)
    int row, col;          // pair indices within the two classes
    double norm;
};

__device__ __forceinline__ JKQuartet jk_quartet_at(const JKSeg& sg, int row, int col) {
    JKQuartet q;
    if (sg.kl_base) col += __ldg(sg.kl_base + row);
    const int bij = sg.pair_ij0 + row, bkl = sg.pair_kl0 + col;
    q.bij = bij;
    q.bkl = bkl;
    q.i0 = __ldg(sg.pao + bij);
    q.j0 = __ldg(sg.pao + sg.npt + bij);
    q.k0 = __ldg(sg.pao + bkl);
    q.l0 = __ldg(sg.pao + sg.npt + bkl);
    q.prim_ij = sg.prim_ij0 + row;  // primitive k at + k * sg.pst_ij
    q.prim_kl = sg.prim_kl0 + col;
    q.row = row;
    q.col = col;
    // 2 pi^3 / sqrt(pi), halved on the ij == kl diagonal (g2e.c:41, g2e.cu:1025)
    q.norm = JK_FAC * (bij == bkl ? 0.5 : 1.0);
    return q;
}

// Output of the ERI-tensor fill (the reference's GINTfill_int2e,
// cuobc/lib/gint/nr_fill_ao_ints.cu:493-549): element (a, b, c, d) of the
// working basis at eri[(a - off[0]) st[0] + (b - off[1]) st[1] + (c - off[2])
// st[2] + (d - off[3]) st[3]].
struct JKFillOut {
    double* eri;
    long long st[4];
    int off[4];
};

// Walks the tasks t = t0, t0 + step, ... of one segment in increasing order,
// keeping the (row, row start, row end) of the last task so that each step
// costs a few comparisons instead of a binary search over the rows.
struct JKTaskCursor {
    int row;
    long long rbeg, rend;
    __device__ __forceinline__ void init(const JKSeg& sg, long long t) {
        row = jk_find_row(sg.qoff, sg.n_ij, t);
        rbeg = __ldg(sg.qoff + row);
        rend = __ldg(sg.qoff + row + 1);
    }
    // column of task t (t not below the previous task)
    __device__ __forceinline__ int seek(const JKSeg& sg, long long t) {
        while (t >= rend) {
            row++;
            rbeg = rend;
            rend = __ldg(sg.qoff + row + 1);
        }
        return (int)(t - rbeg);
    }
};

// Task sources of a launch.  JKOneSeg: one segment passed by value in the
// kernel's parameter space, task count at task0[1].  JKSegTable: several
// segments (one per molecule of a batch) in global memory with exclusive task
// prefix segt[0..nseg]; all segments of a launch share the class and the
// primitive counts.  Cursors walk increasing task indices.
struct JKOneSeg {
    const JKSeg& sg;
    const long long* task0;
    __device__ __forceinline__ long long total() const { return task0[1]; }
    __device__ __forceinline__ unsigned long long* queue() const { return nullptr; }
    __device__ __forceinline__ int grab() const { return 0; }
    __device__ __forceinline__ const JKSeg& first() const { return sg; }
    struct Cursor {
        JKTaskCursor rc;
        __device__ __forceinline__ void init(const JKOneSeg& src, long long t) { rc.init(src.sg, t); }
        // (segment, row, col) of task t
        __device__ __forceinline__ const JKSeg& seek(const JKOneSeg& src, long long t, int& row, int& col) {
            col = rc.seek(src.sg, t);
            row = rc.row;
            return src.sg;
        }
    };
};

// Persistent mode (queue != nullptr): the grid is the resident capacity of
// the device and its warps (thread kernels) or blocks (team and generic
// kernels) take chunks of `grab` consecutive tasks from the device counter
// *queue (zeroed before the launch) until the tasks run out; there is no
// waiting on other blocks, only an atomic add per chunk.  Otherwise the
// tasks are split into equal contiguous chunks over the grid.
struct JKSegTable {
    const JKSeg* segs;
    const long long* segt;
    int nseg;
    unsigned long long* q;
    int g;
    __device__ __forceinline__ long long total() const { return segt[nseg]; }
    __device__ __forceinline__ unsigned long long* queue() const { return q; }
    __device__ __forceinline__ int grab() const { return g; }
    __device__ __forceinline__ const JKSeg& first() const { return segs[0]; }
    struct Cursor {
        int s;
        long long sbeg, send;
        JKTaskCursor rc;
        __device__ __forceinline__ void init(const JKSegTable& src, long long t) {
            s = jk_find_seg(src.segt, src.nseg, t);
            sbeg = src.segt[s];
            send = src.segt[s + 1];
            rc.init(src.segs[s], t - sbeg);
        }
        __device__ __forceinline__ const JKSeg& seek(const JKSegTable& src, long long t, int& row, int& col) {
            if (t >= send) {
                while (t >= src.segt[s + 1]) s++;
                sbeg = src.segt[s];
                send = src.segt[s + 1];
                rc.init(src.segs[s], t - sbeg);
            }
            col = rc.seek(src.segs[s], t - sbeg);
            row = rc.row;
            return src.segs[s];
        }
    };
};

// prefactors of one primitive quartet
struct JKPrim {
    double x, A, B, AB, sy;  // Boys argument, exponent sums, y seed
    double iA, iB, iAB;      // 1/A, 1/B, 1/(A+B)
    double P[3], Q[3];
};

// One primitive pair of a shell pair (exponent sum, its inverse, e12 / a12,
// product centre).  The primitive loops load the ket side once per ket
// primitive pair and pair it with every bra primitive pair (the bra side is
// the same for the lanes of a warp, a broadcast from L1), instead of
// reloading both sides for every primitive quartet.
struct JKPP {
    double a, ia, e, P[3];
};

__device__ __forceinline__ JKPP jk_pp(const JKSeg& sg, int p) {
    JKPP r;
    r.a = __ldg(sg.a12 + p);
    r.ia = __ldg(sg.ia12 + p);
    r.e = __ldg(sg.e12 + p) * r.ia;
    r.P[0] = __ldg(sg.x12 + p);
    r.P[1] = __ldg(sg.y12 + p);
    r.P[2] = __ldg(sg.z12 + p);
    return r;
}

__device__ __forceinline__ JKPrim jk_prim2(const JKPP& b, const JKPP& k) {
    JKPrim p;
    p.A = b.a;
    p.B = k.a;
    p.iA = b.ia;
    p.iB = k.ia;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        p.P[d] = b.P[d];
        p.Q[d] = k.P[d];
    }
    p.AB = p.A + p.B;
    // one reciprocal square root gives both 1/(A+B) and 1/sqrt(A+B)
    const double rs = rsqrt(p.AB);
    p.iAB = rs * rs;
    const double rho = p.A * p.B * p.iAB;
    const double dx = p.P[0] - p.Q[0], dy = p.P[1] - p.Q[1], dz = p.P[2] - p.Q[2];
    p.x = rho * (dx * dx + dy * dy + dz * dz);
    p.sy = b.e * k.e * rs;
    return p;
}

// build the 2D block of (axis d, root r) into out (strides XSI, XSJ of i, j)
template <class C, typename R, int XSI = C::SI, int XSJ = C::SJ, typename OutT>
__device__ __forceinline__ void jk_unit(const JKPrim& p, double s, double w, int d, double norm, const double* ri,
                                        const double* rj, const double* rk, const double* rl, OutT* out) {
    // select by d without dynamic indexing (keeps everything in registers)
#define JK_PICK(a) (d == 0 ? (a)[0] : (d == 1 ? (a)[1] : (a)[2]))
    double siAB = s * p.iAB;
    double bs = p.B * siAB, as = p.A * siAB;
    double b00 = 0.5 * siAB;
    double b10 = 0.5 * p.iA * (1. - bs);
    double b01 = 0.5 * p.iB * (1. - as);
    double Pd = JK_PICK(p.P), Qd = JK_PICK(p.Q);
    double Rid = JK_PICK(ri), Rjd = JK_PICK(rj), Rkd = JK_PICK(rk), Rld = JK_PICK(rl);
    double pq = Pd - Qd;
    double c00 = (Pd - Rid) - bs * pq;
    double c0p = (Qd - Rkd) + as * pq;
    double seed = d == 0 ? norm : (d == 1 ? p.sy : w);
    rys_2d<R, C, XSI, XSJ>((R)seed, (R)c00, (R)c0p, (R)b10, (R)b01, (R)b00, (R)(Rid - Rjd), (R)(Rkd - Rld), out);
}

// ---------------------------------------------------------------------------
// FP32 quartets of the mixed mode at low order: the primitive prefactors,
// the Boys function / Rys nodes and the recursion all in float.  Pair data
// comes from the float copy (JKSeg::pf); P - Q is formed from the small
// differences P - R_i, Q - R_k and the centre difference R_i - R_k (computed
// in double once per contracted quartet) so that it keeps its relative
// precision.
// ---------------------------------------------------------------------------
struct JKPrimF {
    float x, A, B, iA, iB, iAB, sy;
    float PA[3], QC[3], PQ[3];
};

// single-precision primitive pair: a12, 1/a12, e12/a12, P - R of its first shell
struct JKPPF {
    float a, ia, e, D[3];
};

__device__ __forceinline__ JKPPF jk_ppf(const JKSeg& sg, int p) {
    const float* f = sg.pf;
    const long long n = sg.npf;
    JKPPF r;
    r.a = __ldg(f + p);
    r.ia = __ldg(f + n + p);
    r.e = __ldg(f + 2 * n + p);
#pragma unroll
    for (int d = 0; d < 3; d++) r.D[d] = __ldg(f + (3 + d) * n + p);
    return r;
}

__device__ __forceinline__ JKPrimF jk_prim_f2(const JKPPF& b, const JKPPF& k, const float* ac) {
    JKPrimF p;
    p.A = b.a;
    p.B = k.a;
    p.iA = b.ia;
    p.iB = k.ia;
#pragma unroll
    for (int d = 0; d < 3; d++) {
        p.PA[d] = b.D[d];
        p.QC[d] = k.D[d];
        p.PQ[d] = (p.PA[d] - p.QC[d]) + ac[d];
    }
    const float rs = rsqrtf(p.A + p.B);
    p.iAB = rs * rs;
    p.x = p.A * p.B * p.iAB * (p.PQ[0] * p.PQ[0] + p.PQ[1] * p.PQ[1] + p.PQ[2] * p.PQ[2]);
    p.sy = b.e * k.e * rs;
    return p;
}

template <class C, int XSI = C::SI, int XSJ = C::SJ, typename OutT>
__device__ __forceinline__ void jk_unit_f(const JKPrimF& p, float s, float w, int d, float norm, const float* dij,
                                          const float* dkl, OutT* out) {
    float siAB = s * p.iAB;
    float bs = p.B * siAB, as = p.A * siAB;
    float b00 = 0.5f * siAB;
    float b10 = 0.5f * p.iA * (1.f - bs);
    float b01 = 0.5f * p.iB * (1.f - as);
    float pq = JK_PICK(p.PQ);
    float c00 = JK_PICK(p.PA) - bs * pq;
    float c0p = JK_PICK(p.QC) + as * pq;
    float seed = d == 0 ? norm : (d == 1 ? p.sy : w);
    rys_2d<float, C, XSI, XSJ>(seed, c00, c0p, b10, b01, b00, JK_PICK(dij), JK_PICK(dkl), out);
}
#undef JK_PICK

// FP32 primitive path for this class and arithmetic type
template <class C, typename R>
struct JKF32Prim {
    static constexpr bool value = sizeof(R) == 4 && C::NROOTS <= JK_F32_ROOTS;
};

// centres of the two shells of pair p
__device__ __forceinline__ void load_pair_centres(const JKSeg& sg, int p, double* ra, double* rb) {
#pragma unroll
    for (int d = 0; d < 3; d++) {
        ra[d] = __ldg(sg.pgeo + (size_t)d * sg.npt + p);
        rb[d] = __ldg(sg.pgeo + (size_t)(3 + d) * sg.npt + p);
    }
}

// D_ab with the reference's index convention dm[a + nao*b]
#define DM(a, b) __ldg(D + (a) + (size_t)nao * (b))

// ===========================================================================
// P = 0: one thread per quartet.  The Cartesian components are accumulated
// for bra indices ci in [CI0, CI1) per pass; classes too large for one pass
// run NPASS passes over the primitive quartets (the 2D blocks are rebuilt
// per pass, the accumulators of one pass only are live).
// ===========================================================================
// ---------------------------------------------------------------------------
// Digestion of one quartet's Cartesian block (bra components ci in
// [CI0, CI0 + NI)) into J and K through a sink:
//   J_ij += (ij|kl) D_kl, J_kl += (ij|kl) D_ij,
//   K_ik += (ij|kl) D_jl, K_il += (ij|kl) D_jk, K_jk += (ij|kl) D_il,
//   K_jl += (ij|kl) D_ik
// (cuobc/lib/gvhf/contract_jk.cu:225-316).  JKSinkGlobal adds every element
// to the output buffers with one global atomic, element (a, b) at a + nao*b;
// JKSinkSmem adds into the shared-memory blocks of a tile.
// ---------------------------------------------------------------------------
struct JKSinkGlobal {
    double* vj;
    double* vk;
    int nao;
    size_t nn;
    __device__ __forceinline__ void jij(int idm, int a, int b, double v) const {
        atomicAdd(vj + idm * nn + a + (size_t)nao * b, v);
    }
    __device__ __forceinline__ void jkl(int idm, int a, int b, double v) const {
        atomicAdd(vj + idm * nn + a + (size_t)nao * b, v);
    }
    __device__ __forceinline__ void kik(int idm, int a, int b, double v) const {
        atomicAdd(vk + idm * nn + a + (size_t)nao * b, v);
    }
    __device__ __forceinline__ void kil(int idm, int a, int b, double v) const { kik(idm, a, b, v); }
    __device__ __forceinline__ void kjk(int idm, int a, int b, double v) const { kik(idm, a, b, v); }
    __device__ __forceinline__ void kjl(int idm, int a, int b, double v) const { kik(idm, a, b, v); }
};

__device__ __forceinline__ JKSinkGlobal jk_sink_global(const JKSeg& sg) {
    return JKSinkGlobal{sg.vj, sg.vk, sg.nao, (size_t)sg.nao * sg.nao};
}

template <class C, typename R, int NI, class Sink>
__device__ __forceinline__ void jk_thread_digest(const JKSeg& sg, const JKQuartet& q, int CI0, const R* acc,
                                                 const Sink& sink) {
    const int nao = sg.nao;
    const int i0 = q.i0 + CI0, j0 = q.j0;
    const int k0 = q.k0, l0 = q.l0;
    // the lanes of a warp usually share the ij pair (consecutive kl of one
    // row): then the J_ij block is summed over the warp before it is added.
    // In a batched launch a warp can straddle two molecules whose pairs
    // carry the same indices, so the lanes must also share the output.
    const unsigned am = __activemask();
    bool wsame = false;
    if (am == 0xffffffffu) {
        const unsigned long long out = (unsigned long long)(sg.jp_ij ? (const void*)sg.jp_ij : (const void*)sg.vj);
        const int p_0 = __shfl_sync(am, q.bij, 0);
        unsigned long long o_0 = __shfl_sync(am, out, 0);
        wsame = __all_sync(am, q.bij == p_0 && out == o_0);
    }
#define ACC(i, j, k, l) ((double)acc[(((i) * C::NFJ + (j)) * C::NFK + (k)) * C::NFL + (l)])
    for (int idm = 0; idm < sg.n_dm; idm++) {
        const double* D = sg.dm + (size_t)idm * nao * nao;
        if (sg.vj && sg.dp_ij) {
            // pair-packed: consecutive lanes hold consecutive kl pairs, so the
            // D_kl loads and the J_kl additions are coalesced
            const size_t po = (size_t)idm * sg.pk_stride;
            const double* Dij = sg.dp_ij + po + q.row;
            const double* Dkl = sg.dp_kl + po + q.col;
#pragma unroll
            for (int i = 0; i < NI; i++)
#pragma unroll
                for (int j = 0; j < C::NFJ; j++) {
                    double v = 0;
#pragma unroll
                    for (int k = 0; k < C::NFK; k++)
#pragma unroll
                        for (int l = 0; l < C::NFL; l++)
                            v += ACC(i, j, k, l) * __ldg(Dkl + (size_t)(k * C::NFL + l) * sg.np_kl);
                    double* J = sg.jp_ij + po + (size_t)((CI0 + i) * C::NFJ + j) * sg.np_ij + q.row;
                    if (wsame) {
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                        if ((threadIdx.x & 31) == 0) atomicAdd(J, v);
                    } else {
                        atomicAdd(J, v);
                    }
                }
#pragma unroll
            for (int k = 0; k < C::NFK; k++)
#pragma unroll
                for (int l = 0; l < C::NFL; l++) {
                    double v = 0;
#pragma unroll
                    for (int i = 0; i < NI; i++)
#pragma unroll
                        for (int j = 0; j < C::NFJ; j++)
                            v += ACC(i, j, k, l) * __ldg(Dij + (size_t)((CI0 + i) * C::NFJ + j) * sg.np_ij);
                    atomicAdd(sg.jp_kl + po + (size_t)(k * C::NFL + l) * sg.np_kl + q.col, v);
                }
        } else if (sg.vj) {
#pragma unroll
            for (int i = 0; i < NI; i++)
#pragma unroll
                for (int j = 0; j < C::NFJ; j++) {
                    double v = 0;
#pragma unroll
                    for (int k = 0; k < C::NFK; k++)
#pragma unroll
                        for (int l = 0; l < C::NFL; l++) v += ACC(i, j, k, l) * DM(k0 + k, l0 + l);
                    if (wsame) {
#pragma unroll
                        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
                        if ((threadIdx.x & 31) == 0) sink.jij(idm, i0 + i, j0 + j, v);
                    } else {
                        sink.jij(idm, i0 + i, j0 + j, v);
                    }
                }
#pragma unroll
            for (int k = 0; k < C::NFK; k++)
#pragma unroll
                for (int l = 0; l < C::NFL; l++) {
                    double v = 0;
#pragma unroll
                    for (int i = 0; i < NI; i++)
#pragma unroll
                        for (int j = 0; j < C::NFJ; j++) v += ACC(i, j, k, l) * DM(i0 + i, j0 + j);
                    sink.jkl(idm, k0 + k, l0 + l, v);
                }
        }
        if (sg.vk) {
#pragma unroll
            for (int i = 0; i < NI; i++)
#pragma unroll
                for (int k = 0; k < C::NFK; k++) {
                    double v = 0;
#pragma unroll
                    for (int j = 0; j < C::NFJ; j++)
#pragma unroll
                        for (int l = 0; l < C::NFL; l++) v += ACC(i, j, k, l) * DM(l0 + l, j0 + j);
                    sink.kik(idm, i0 + i, k0 + k, v);
                }
#pragma unroll
            for (int i = 0; i < NI; i++)
#pragma unroll
                for (int l = 0; l < C::NFL; l++) {
                    double v = 0;
#pragma unroll
                    for (int j = 0; j < C::NFJ; j++)
#pragma unroll
                        for (int k = 0; k < C::NFK; k++) v += ACC(i, j, k, l) * DM(k0 + k, j0 + j);
                    sink.kil(idm, i0 + i, l0 + l, v);
                }
#pragma unroll
            for (int j = 0; j < C::NFJ; j++)
#pragma unroll
                for (int k = 0; k < C::NFK; k++) {
                    double v = 0;
#pragma unroll
                    for (int i = 0; i < NI; i++)
#pragma unroll
                        for (int l = 0; l < C::NFL; l++) v += ACC(i, j, k, l) * DM(l0 + l, i0 + i);
                    sink.kjk(idm, j0 + j, k0 + k, v);
                }
#pragma unroll
            for (int j = 0; j < C::NFJ; j++)
#pragma unroll
                for (int l = 0; l < C::NFL; l++) {
                    double v = 0;
#pragma unroll
                    for (int i = 0; i < NI; i++)
#pragma unroll
                        for (int k = 0; k < C::NFK; k++) v += ACC(i, j, k, l) * DM(k0 + k, i0 + i);
                    sink.kjl(idm, j0 + j, l0 + l, v);
                }
        }
    }
#undef ACC
}

// acc[i][j][k][l] += Ix Iy Iz for the bra components ci in [CI0, CI0 + NI)
template <class C, typename R, int CI0, int NI>
__device__ __forceinline__ void jk_thread_products(R* acc, const R* Ix, const R* Iy, const R* Iz) {
#pragma unroll
    for (int i = 0; i < NI; i++)
#pragma unroll
        for (int j = 0; j < C::NFJ; j++)
#pragma unroll
            for (int k = 0; k < C::NFK; k++)
#pragma unroll
                for (int l = 0; l < C::NFL; l++) {
                    int ox = cart_lx(C::LI, CI0 + i) * C::SI + cart_lx(C::LJ, j) * C::SJ + cart_lx(C::LK, k) * C::SK +
                             cart_lx(C::LL, l);
                    int oy = cart_ly(C::LI, CI0 + i) * C::SI + cart_ly(C::LJ, j) * C::SJ + cart_ly(C::LK, k) * C::SK +
                             cart_ly(C::LL, l);
                    int oz = cart_lz(C::LI, CI0 + i) * C::SI + cart_lz(C::LJ, j) * C::SJ + cart_lz(C::LK, k) * C::SK +
                             cart_lz(C::LL, l);
                    acc[((i * C::NFJ + j) * C::NFK + k) * C::NFL + l] += Ix[ox] * Iy[oy] * Iz[oz];
                }
}

template <class C, typename R, int CI0, int CI1, class Sink>
__device__ __forceinline__ void jk_thread_pass(const JKSeg& sg, const JKQuartet& q, const double* __restrict__ tab,
                                               const double* ri, const double* rj, const double* rk,
                                               const double* rl, const Sink& sink, const JKFillOut* fo) {
    constexpr int NR = C::NROOTS;
    constexpr int NI = CI1 - CI0;
    constexpr int NA = NI * C::NFJ * C::NFK * C::NFL;
    R acc[NA];
#pragma unroll
    for (int e = 0; e < NA; e++) acc[e] = R(0);
    if constexpr (JKF32Prim<C, R>::value) {
        const float* tabf = reinterpret_cast<const float*>(tab);
        float dij[3], dkl[3], ac[3];
#pragma unroll
        for (int d = 0; d < 3; d++) {
            dij[d] = (float)(ri[d] - rj[d]);
            dkl[d] = (float)(rk[d] - rl[d]);
            ac[d] = (float)(ri[d] - rk[d]);
        }
        const float normf = (float)q.norm;
        const int npij = sg.pnp ? __ldg(sg.pnp + q.bij) : sg.nprim_ij;
        const int npkl = sg.pnp ? __ldg(sg.pnp + q.bkl) : sg.nprim_kl;
        JKPPF kn = jk_ppf(sg, q.prim_kl);
        for (int kp = 0; kp < npkl; kp++) {
            const JKPPF kc = kn;
            if (kp + 1 < npkl) kn = jk_ppf(sg, q.prim_kl + (kp + 1) * sg.pst_kl);  // next ket primitive, in flight
            for (int ip = 0; ip < npij; ip++) {
                JKPrimF p = jk_prim_f2(jk_ppf(sg, q.prim_ij + ip * sg.pst_ij), kc, ac);
                float rs[NR], rw[NR];
                rys_roots_all_f<NR>(tabf, p.x, rs, rw);
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    float Ix[C::GS], Iy[C::GS], Iz[C::GS];
                    jk_unit_f<C>(p, rs[r], rw[r], 0, normf, dij, dkl, Ix);
                    jk_unit_f<C>(p, rs[r], rw[r], 1, normf, dij, dkl, Iy);
                    jk_unit_f<C>(p, rs[r], rw[r], 2, normf, dij, dkl, Iz);
                    jk_thread_products<C, R, CI0, NI>(acc, Ix, Iy, Iz);
                }
            }
        }
    } else {
        const int npij = sg.pnp ? __ldg(sg.pnp + q.bij) : sg.nprim_ij;
        const int npkl = sg.pnp ? __ldg(sg.pnp + q.bkl) : sg.nprim_kl;
        JKPP kn = jk_pp(sg, q.prim_kl);
        for (int kp = 0; kp < npkl; kp++) {
            const JKPP kc = kn;
            if (kp + 1 < npkl) kn = jk_pp(sg, q.prim_kl + (kp + 1) * sg.pst_kl);  // next ket primitive, in flight
            for (int ip = 0; ip < npij; ip++) {
                JKPrim p = jk_prim2(jk_pp(sg, q.prim_ij + ip * sg.pst_ij), kc);
                double rs[NR], rw[NR];
                rys_roots_all<NR>(tab, p.x, rs, rw);
#pragma unroll
                for (int r = 0; r < NR; r++) {
                    const double s = rs[r], w = rw[r];
                    R Ix[C::GS], Iy[C::GS], Iz[C::GS];
                    jk_unit<C, R>(p, s, w, 0, q.norm, ri, rj, rk, rl, Ix);
                    jk_unit<C, R>(p, s, w, 1, q.norm, ri, rj, rk, rl, Iy);
                    jk_unit<C, R>(p, s, w, 2, q.norm, ri, rj, rk, rl, Iz);
                    jk_thread_products<C, R, CI0, NI>(acc, Ix, Iy, Iz);
                }
            }
        }
    }
    if (fo) {  // ERI-tensor fill: the quartet's block goes to the tensor
        const long long b0 = (long long)(q.i0 + CI0 - fo->off[0]) * fo->st[0] +
                             (long long)(q.j0 - fo->off[1]) * fo->st[1] + (long long)(q.k0 - fo->off[2]) * fo->st[2] +
                             (long long)(q.l0 - fo->off[3]) * fo->st[3];
#pragma unroll
        for (int i = 0; i < NI; i++)
#pragma unroll
            for (int j = 0; j < C::NFJ; j++)
#pragma unroll
                for (int k = 0; k < C::NFK; k++)
#pragma unroll
                    for (int l = 0; l < C::NFL; l++)
                        atomicAdd(fo->eri + b0 + i * fo->st[0] + j * fo->st[1] + k * fo->st[2] + l * fo->st[3],
                                  (double)acc[((i * C::NFJ + j) * C::NFK + k) * C::NFL + l]);
        return;
    }
    jk_thread_digest<C, R, NI>(sg, q, CI0, acc, sink);
}


template <class C, typename R, int PASS, class Sink>
__device__ __forceinline__ void jk_thread_passes(const JKSeg& sg, const JKQuartet& q, const double* __restrict__ tab,
                                                 const double* ri, const double* rj, const double* rk,
                                                 const double* rl, const Sink& sink, const JKFillOut* fo) {
    constexpr int CI0 = PASS * C::GI;
    if constexpr (CI0 < C::NFI) {
        constexpr int CI1 = CI0 + C::GI < C::NFI ? CI0 + C::GI : C::NFI;
        jk_thread_pass<C, R, CI0, CI1>(sg, q, tab, ri, rj, rk, rl, sink, fo);
        jk_thread_passes<C, R, PASS + 1>(sg, q, tab, ri, rj, rk, rl, sink, fo);
    }
}

template <class C, typename R, class Sink>
__device__ __forceinline__ void jk_thread_quartet(const JKSeg& sg, const JKQuartet& q, const double* __restrict__ tab,
                                                  const Sink& sink, const JKFillOut* fo = nullptr) {
    double ri[3], rj[3], rk[3], rl[3];
    load_pair_centres(sg, q.bij, ri, rj);
    load_pair_centres(sg, q.bkl, rk, rl);
    jk_thread_passes<C, R, 0>(sg, q, tab, ri, rj, rk, rl, sink, fo);
}

// Resident 128-thread blocks asked of the register allocator (single-segment
// kernel).  The FP32 quartets hold half-width values and spend more of their
// time waiting on loads, so they get more resident warps; the batched kernel
// keeps C::MINB (its segment cursor would spill).
template <class C, typename R>
struct JKThreadMinBlocks {
    static constexpr int value = sizeof(R) == 4 ? (C::W <= 24 ? 8 : (C::W <= 40 ? 6 : 4)) : C::MINB;
};

template <class C, typename R, class Src>
__device__ __forceinline__ void jk_thread_body(const Src& src, double* jk_tab, const JKFillOut* fo = nullptr) {
    // each warp takes a contiguous chunk of tasks (a multiple of 32); lane i
    // does tasks i, i+32, ... of it, so a warp covers consecutive kl of a row
    const long long total = src.total();
    const int lane = threadIdx.x & 31;
    const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
    const long long wid = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    unsigned long long* queue = src.queue();
    const long long chunk = queue ? (long long)src.grab() : (((total + nwarps - 1) / nwarps) + 31) & ~31LL;
    // static chunks: the grid is sized for the unscreened task count, and a
    // block without any screened task leaves before it loads the Rys table
    // (block-uniform test)
    if (!queue && (long long)blockIdx.x * (blockDim.x >> 5) * chunk >= total) return;
    if (queue && total == 0) return;
    if constexpr (JKF32Prim<C, R>::value)
        rys_table_to_smem_f<C::NROOTS>(src.first().rys, reinterpret_cast<float*>(jk_tab));
    else
        rys_table_to_smem<C::NROOTS>(src.first().rys, jk_tab);
    __syncthreads();
    long long c0 = wid * chunk;
    for (;;) {
        if (queue) {
            unsigned long long g = 0;
            if (lane == 0) g = atomicAdd(queue, (unsigned long long)chunk);
            c0 = (long long)__shfl_sync(0xffffffffu, g, 0);
        }
        if (c0 >= total) break;
        long long t = c0 + lane;
        const long long tend = min(total, c0 + chunk);
        if (t < tend) {
            typename Src::Cursor cur;
            cur.init(src, t);
            for (; t < tend; t += 32) {
                int row, col;
                const JKSeg& sg = cur.seek(src, t, row, col);
                JKQuartet q = jk_quartet_at(sg, row, col);
                if (fo) q.norm = JK_FAC;  // the fill has no 1/2 on the ij == kl diagonal
                jk_thread_quartet<C, R>(sg, q, jk_tab, jk_sink_global(sg), fo);
            }
        }
        if (!queue) break;
    }
}

template <class C, typename R>
__global__ void __launch_bounds__(128, (JKThreadMinBlocks<C, R>::value)) jk_thread_kernel(const __grid_constant__ JKSeg sg,
                                                                 const long long* __restrict__ task0) {
    extern __shared__ __align__(16) double jk_tab[];
    JKOneSeg src{sg, task0};
    jk_thread_body<C, R>(src, jk_tab);
}

// ERI-tensor fill with the thread kernel's register recursion (FP64)
template <class C>
__global__ void __launch_bounds__(128, C::MINB) jk_thread_fill_kernel(const __grid_constant__ JKSeg sg,
                                                                      const long long* __restrict__ task0,
                                                                      const __grid_constant__ JKFillOut out) {
    extern __shared__ __align__(16) double jk_tab[];
    JKOneSeg src{sg, task0};
    jk_thread_body<C, double>(src, jk_tab, &out);
}

template <class C, typename R>
__global__ void __launch_bounds__(128, C::MINB) jk_thread_kernel_batch(const JKSeg* __restrict__ segs,
                                                                       const long long* __restrict__ segt,
                                                                       int nseg, unsigned long long* queue,
                                                                       int grab) {
    extern __shared__ __align__(16) double jk_tab[];
    JKSegTable src{segs, segt, nseg, queue, grab};
    jk_thread_body<C, R>(src, jk_tab);
}

// ===========================================================================
// P > 0: a team of T threads per quartet, teams packed into a block
// ===========================================================================
template <class C>
struct JKTeamShape {
    static constexpr int QPB = (C::T >= 128) ? 1 : (128 / C::T);  // quartets per block
    static constexpr int THREADS = QPB * C::T;
    static constexpr int BWORDS_RAW = C::NFI * C::NFJ + C::NFK * C::NFL + C::NFI * C::NFK + C::NFI * C::NFL +
                                      C::NFJ * C::NFK + C::NFJ * C::NFL;  // digestion buffers
    static constexpr int BWORDS = BWORDS_RAW | 1;
    // per-thread partial J/K blocks of the digestion (reuse the 2D-block space)
    static constexpr int NKET = C::NFK * C::NFL;
    static constexpr int PSTRIDE = C::P == 1 ? NKET + C::NFJ * C::NFK + C::NFJ * C::NFL
                                             : NKET + 2 * C::NFK + 2 * C::NFL;  // doubles per thread
    static constexpr int PWORDS = C::T * PSTRIDE;
    // the Rys table goes to shared memory for up to 4 roots; beyond that the
    // units read the global copy (it would cost 37-60 KB per block)
    static constexpr bool SMEM_TAB = C::NROOTS <= 4;
    static constexpr int TAB = SMEM_TAB ? RysS<C::NROOTS>::WORDS : 0;  // doubles, first in shared memory
    static constexpr int OFF_JIJ = 0, OFF_JKL = OFF_JIJ + C::NFI * C::NFJ, OFF_KIK = OFF_JKL + C::NFK * C::NFL,
                         OFF_KIL = OFF_KIK + C::NFI * C::NFK, OFF_KJK = OFF_KIL + C::NFI * C::NFL,
                         OFF_KJL = OFF_KJK + C::NFJ * C::NFK;
};

// ---------------------------------------------------------------------------
// Shared-memory layout of a team's 2D blocks, padded against bank conflicts.
// Two access patterns dominate: the products, where the thread owning bra
// component ci (and cj) reads element own + o of every block with
// own = lx(ci)*SI (+ lx(cj)*SJ) and o the same for the whole warp; and the
// construction, where lane u writes element idx of unit u at u*GS + idx.  SI
// (and SJ) are padded so that the owned offsets of a team fall in distinct
// banks, GS is odd, and the team stride (the region of one team, which also
// holds the digestion partials) is chosen modulo the bank count so that the
// teams sharing a warp stay apart.  The choice is made at compile time with a
// model of one warp access: the largest number of distinct addresses that
// fall in one bank (bank = element index mod 128 / sizeof(R)).
// ---------------------------------------------------------------------------
constexpr int jk_bank_ways(const int* a, int n, int nb) {
    int cnt[32] = {};
    for (int i = 0; i < n; i++) {
        bool dup = false;
        for (int j = 0; j < i; j++)
            if (a[j] == a[i]) {
                dup = true;
                break;
            }
        if (!dup) cnt[a[i] % nb]++;
    }
    int w = 0;
    for (int b = 0; b < nb; b++) w = cnt[b] > w ? cnt[b] : w;
    return w;
}

template <class C>
constexpr int jk_team_own(int lane, int d, int si, int sj) {
    const int ci = C::P == 1 ? lane : lane / C::NFJ;
    const int cj = C::P == 1 ? 0 : lane - ci * C::NFJ;
    const int ei = d == 0 ? cart_lx(C::LI, ci) : (d == 1 ? cart_ly(C::LI, ci) : cart_lz(C::LI, ci));
    const int ej = C::P == 1 ? 0 : (d == 0 ? cart_lx(C::LJ, cj) : (d == 1 ? cart_ly(C::LJ, cj) : cart_lz(C::LJ, cj)));
    return ei * si + ej * sj;
}

// distinct-bank spread of the owned offsets of one team (worst multiplicity)
template <class C>
constexpr int jk_team_own_ways(int si, int sj, int nb) {
    int a[32] = {};
    int n = 0;
    for (int x = 0; x <= C::LI; x++)
        for (int y = 0; y <= (C::P == 2 ? C::LJ : 0); y++) a[n++] = x * si + y * sj;
    return jk_bank_ways(a, n, nb);
}

// bank ways summed over the warps of a block: three product reads (x, y, z
// offsets) and one construction write per warp
template <class C>
constexpr int jk_team_ways(int si, int sj, int gs, int reg, int nb, int threads) {
    int a[32] = {};
    int total = 0;
    for (int w = 0; w * 32 < threads; w++) {
        const int t1 = threads < w * 32 + 32 ? threads : w * 32 + 32;
        for (int d = 0; d < 3; d++) {
            int n = 0;
            for (int t = w * 32; t < t1; t++) a[n++] = (t / C::T) * reg + jk_team_own<C>(t % C::T, d, si, sj);
            total += jk_bank_ways(a, n, nb);
        }
        int n = 0;
        for (int t = w * 32; t < t1; t++)
            if (t % C::T < 3 * C::NROOTS) a[n++] = (t / C::T) * reg + (t % C::T) * gs;
        if (n) total += jk_bank_ways(a, n, nb);
    }
    return total;
}

template <class C>
constexpr int jk_team_pick_si(int sj, int nb) {
    const int s0 = C::P == 2 ? C::LJ * sj + C::SJ : C::SI;  // blocks of i do not overlap
    int best = s0, bw = 1 << 20;
    for (int s = s0; s < s0 + nb; s++) {
        const int w = jk_team_own_ways<C>(s, sj, nb);
        if (w < bw) {
            bw = w;
            best = s;
        }
    }
    return best;
}

template <class C>
constexpr int jk_team_pick_words(int si, int sj, int gs, int words0, int esize, int threads) {
    int best = words0, bw = 1 << 20;
    for (int r = 0; r < 16; r++) {
        const int words = words0 + ((r - words0 % 16) + 16) % 16;
        const int w = jk_team_ways<C>(si, sj, gs, words * 8 / esize, 128 / esize, threads);
        if (w < bw) {
            bw = w;
            best = words;
        }
    }
    return best;
}

template <class C, typename R>
struct JKTeamLayout {
    using S = JKTeamShape<C>;
    static constexpr int NB = 128 / (int)sizeof(R);  // banks in elements of R
    static constexpr int SJ = C::P == 2 ? (C::SJ | 1) : C::SJ;
    static constexpr int SI = jk_team_pick_si<C>(SJ, NB);
    static constexpr int GS = (C::LI * SI + C::LJ * SJ + (C::LK + 1) * (C::LL + 1)) | 1;  // elements per unit
    // region of one team in doubles: the 2D blocks of all roots or the digestion partials
    static constexpr int GW = (3 * C::NROOTS * GS * (int)sizeof(R) + 7) / 8;
    static constexpr int WORDS0 = GW > S::PWORDS ? GW : S::PWORDS;
    static constexpr int WORDS = jk_team_pick_words<C>(SI, SJ, GS, WORDS0, (int)sizeof(R), S::THREADS);
};

// bytes per team of the region shared by the 2D blocks and the digestion
// partials
template <class C, typename R>
__host__ __device__ constexpr size_t jk_team_region() {
    return (size_t)JKTeamLayout<C, R>::WORDS * 8;
}

template <class C, typename R>
__host__ __device__ constexpr size_t jk_team_gbytes() {
    using S = JKTeamShape<C>;
    return ((size_t)S::QPB * jk_team_region<C, R>() + 15) & ~(size_t)15;
}

template <class C, typename R>
__host__ __device__ constexpr size_t jk_team_smem() {
    using S = JKTeamShape<C>;
    return (size_t)S::TAB * sizeof(double) + jk_team_gbytes<C, R>() + (size_t)S::QPB * S::BWORDS * sizeof(double);
}

template <class C, typename R, class Src>
__device__ __forceinline__ void jk_team_body(const Src& src, const JKFillOut* fo = nullptr) {
    using S = JKTeamShape<C>;
    using L = JKTeamLayout<C, R>;
    constexpr int T = C::T, NR = C::NROOTS;
    extern __shared__ __align__(16) unsigned char jk_smem[];
    const int team = threadIdx.x / T, lane = threadIdx.x - team * T;
    double* tab = reinterpret_cast<double*>(jk_smem);
    unsigned char* gbase = jk_smem + (size_t)S::TAB * sizeof(double);
    R* g = reinterpret_cast<R*>(gbase + (size_t)team * jk_team_region<C, R>());
    double* part = reinterpret_cast<double*>(g);  // digestion partials reuse the 2D-block space
    double* buf = reinterpret_cast<double*>(gbase + jk_team_gbytes<C, R>()) + (size_t)team * S::BWORDS;
    const JKSeg& sg0 = src.first();
    // each team takes a contiguous chunk of tasks; every team of the block
    // runs the same number of iterations (the block synchronises inside).
    // The grid is sized for the unscreened task count: a block whose first
    // team has no screened task leaves before it loads the Rys table.
    const long long total = src.total();
    const long long nteams = (long long)gridDim.x * S::QPB;
    unsigned long long* queue = src.queue();
    // tasks per team and round: the whole static chunk, or one grab of the
    // persistent mode (a block takes QPB grabs at once)
    const long long chunk = queue ? (long long)src.grab() : (total + nteams - 1) / nteams;
    if (!queue && (long long)blockIdx.x * S::QPB * chunk >= total) return;
    if (queue && total == 0) return;
    // FP32 quartets at low order: float prefactors, nodes and weights (the
    // table copy in shared memory is then single precision)
    constexpr bool F32P = JKF32Prim<C, R>::value && S::SMEM_TAB;
    if (S::SMEM_TAB) {
        if constexpr (F32P) rys_table_to_smem_f<NR>(sg0.rys, reinterpret_cast<float*>(tab));
        else rys_table_to_smem<NR>(sg0.rys, tab);
    }

    // owned Cartesian indices
    int ci = 0, cj = 0;
    if (C::P == 1) ci = lane;
    if (C::P == 2) {
        ci = lane / C::NFJ;
        cj = lane - ci * C::NFJ;
    }
    int own_x = cart_lx(C::LI, ci) * L::SI, own_y = cart_ly(C::LI, ci) * L::SI, own_z = cart_lz(C::LI, ci) * L::SI;
    if (C::P == 2) {
        own_x += cart_lx(C::LJ, cj) * L::SJ;
        own_y += cart_ly(C::LJ, cj) * L::SJ;
        own_z += cart_lz(C::LJ, cj) * L::SJ;
    }

    __syncthreads();
    const int nprim_ij = sg0.nprim_ij, nprim_kl = sg0.nprim_kl;  // uniform within a launch
    __shared__ long long s_grab;
    long long bbase = (long long)blockIdx.x * S::QPB * chunk;
    for (;;) {
    if (queue) {
        __syncthreads();  // the previous round's readers of s_grab are done
        if (threadIdx.x == 0) s_grab = (long long)atomicAdd(queue, (unsigned long long)(chunk * S::QPB));
        __syncthreads();
        bbase = s_grab;
        if (bbase >= total) break;  // block-uniform
    }
    const long long tbeg = bbase + team * chunk, tend = min(total, tbeg + chunk);
    typename Src::Cursor cur;
    if (tbeg < tend) cur.init(src, tbeg);
    for (long long it = 0; it < chunk; it++) {
        const long long t = tbeg + it;
        const bool active = t < tend;
        JKQuartet q;
        double ri[3], rj[3], rk[3], rl[3];
        const JKSeg* sgp = &sg0;
        if (active) {
            int row, col;
            sgp = &cur.seek(src, t, row, col);
            q = jk_quartet_at(*sgp, row, col);
            if (fo) q.norm = JK_FAC;  // the fill has no 1/2 on the ij == kl diagonal
        }
        const JKSeg& sg = *sgp;
        if (active) {
            load_pair_centres(sg, q.bij, ri, rj);
            load_pair_centres(sg, q.bkl, rk, rl);
        }
        R acc[C::NACC];
#pragma unroll
        for (int e = 0; e < C::NACC; e++) acc[e] = R(0);
        float dijf[3], dklf[3], acf[3];
        if (F32P && active) {
#pragma unroll
            for (int d = 0; d < 3; d++) {
                dijf[d] = (float)(ri[d] - rj[d]);
                dklf[d] = (float)(rk[d] - rl[d]);
                acf[d] = (float)(ri[d] - rk[d]);
            }
        }
        for (int kp = 0; kp < nprim_kl; kp++) {
            JKPP kc;
            JKPPF kcf;
            if (active) {
                if constexpr (F32P) kcf = jk_ppf(sg, q.prim_kl + kp * sg.pst_kl);
                else kc = jk_pp(sg, q.prim_kl + kp * sg.pst_kl);
            }
            for (int ip = 0; ip < nprim_ij; ip++) {
                if (active) {
                    if constexpr (F32P) {
                        const JKPrimF pf = jk_prim_f2(jk_ppf(sg, q.prim_ij + ip * sg.pst_ij), kcf, acf);
                        const float normf = (float)q.norm;
                        for (int u = lane; u < 3 * NR; u += T) {
                            int r = u / 3, d = u - 3 * r;
                            float s, w;
                            rys_root_one_f<NR>(reinterpret_cast<const float*>(tab), pf.x, r, s, w);
                            jk_unit_f<C, L::SI, L::SJ>(pf, s, w, d, normf, dijf, dklf, g + u * L::GS);
                        }
                    } else {
                        JKPrim p = jk_prim2(jk_pp(sg, q.prim_ij + ip * sg.pst_ij), kc);
                        for (int u = lane; u < 3 * NR; u += T) {
                            int r = u / 3, d = u - 3 * r;
                            double s, w;
                            if (S::SMEM_TAB) rys_root_one<NR>(tab, p.x, r, s, w);
                            else rys_root<NR>(sg.rys, p.x, r, s, w);
                            jk_unit<C, R, L::SI, L::SJ>(p, s, w, d, q.norm, ri, rj, rk, rl, g + u * L::GS);
                        }
                    }
                }
                __syncthreads();
                if (active) {
#pragma unroll
                    for (int r = 0; r < NR; r++) {
                        const R* gx = g + (3 * r) * L::GS;
                        const R* gy = gx + L::GS;
                        const R* gz = gy + L::GS;
                        if (C::P == 1) {
#pragma unroll
                            for (int j = 0; j < C::NFJ; j++)
#pragma unroll
                                for (int k = 0; k < C::NFK; k++)
#pragma unroll
                                    for (int l = 0; l < C::NFL; l++) {
                                        int ox = cart_lx(C::LJ, j) * L::SJ + cart_lx(C::LK, k) * C::SK + cart_lx(C::LL, l);
                                        int oy = cart_ly(C::LJ, j) * L::SJ + cart_ly(C::LK, k) * C::SK + cart_ly(C::LL, l);
                                        int oz = cart_lz(C::LJ, j) * L::SJ + cart_lz(C::LK, k) * C::SK + cart_lz(C::LL, l);
                                        acc[(j * C::NFK + k) * C::NFL + l] +=
                                            gx[own_x + ox] * gy[own_y + oy] * gz[own_z + oz];
                                    }
                        } else {
#pragma unroll
                            for (int k = 0; k < C::NFK; k++)
#pragma unroll
                                for (int l = 0; l < C::NFL; l++) {
                                    int ox = cart_lx(C::LK, k) * C::SK + cart_lx(C::LL, l);
                                    int oy = cart_ly(C::LK, k) * C::SK + cart_ly(C::LL, l);
                                    int oz = cart_lz(C::LK, k) * C::SK + cart_lz(C::LL, l);
                                    acc[k * C::NFL + l] += gx[own_x + ox] * gy[own_y + oy] * gz[own_z + oz];
                                }
                        }
                    }
                }
                __syncthreads();
            }
        }

        if (fo) {  // ERI-tensor fill: each thread writes its owned components
            if (active) {
                const long long b0 = (long long)(q.i0 + ci - fo->off[0]) * fo->st[0] +
                                     (long long)(q.j0 + cj - fo->off[1]) * fo->st[1] +
                                     (long long)(q.k0 - fo->off[2]) * fo->st[2] +
                                     (long long)(q.l0 - fo->off[3]) * fo->st[3];
                if (C::P == 1) {
#pragma unroll
                    for (int j = 0; j < C::NFJ; j++)
#pragma unroll
                        for (int k = 0; k < C::NFK; k++)
#pragma unroll
                            for (int l = 0; l < C::NFL; l++)
                                atomicAdd(fo->eri + b0 + j * fo->st[1] + k * fo->st[2] + l * fo->st[3],
                                          (double)acc[(j * C::NFK + k) * C::NFL + l]);
                } else {
#pragma unroll
                    for (int k = 0; k < C::NFK; k++)
#pragma unroll
                        for (int l = 0; l < C::NFL; l++)
                            atomicAdd(fo->eri + b0 + k * fo->st[2] + l * fo->st[3], (double)acc[k * C::NFL + l]);
                }
            }
            continue;
        }
        // ---- digestion ----
        // Outputs a thread owns completely go to buf; the others are written as
        // per-thread partials (no shared atomics), summed by the team after a
        // barrier, then every element is flushed with one global atomic.
        const int n_dm = sg.n_dm;
        for (int idm = 0; idm < n_dm; idm++) {
            // every element of buf is written below before it is flushed
            double* mine = part + (size_t)lane * S::PSTRIDE;
            if (active) {
                const int nao = sg.nao;
                const int i0 = q.i0, j0 = q.j0;
                const int k0 = q.k0, l0 = q.l0;
                const double* D = sg.dm + (size_t)idm * nao * nao;
                if (C::P == 1) {
#define A1(j, k, l) ((double)acc[((j) * C::NFK + (k)) * C::NFL + (l)])
                    const int I = i0 + ci;
                    double* pjkl = mine;
                    double* pkjk = mine + S::NKET;
                    double* pkjl = pkjk + C::NFJ * C::NFK;
                    if (sg.vj) {
#pragma unroll
                        for (int j = 0; j < C::NFJ; j++) {  // J_ij: complete in-thread
                            double v = 0;
#pragma unroll
                            for (int k = 0; k < C::NFK; k++)
#pragma unroll
                                for (int l = 0; l < C::NFL; l++) v += A1(j, k, l) * DM(k0 + k, l0 + l);
                            buf[S::OFF_JIJ + ci * C::NFJ + j] = v;
                        }
#pragma unroll
                        for (int k = 0; k < C::NFK; k++)  // J_kl: partial over i
#pragma unroll
                            for (int l = 0; l < C::NFL; l++) {
                                double v = 0;
#pragma unroll
                                for (int j = 0; j < C::NFJ; j++) v += A1(j, k, l) * DM(I, j0 + j);
                                pjkl[k * C::NFL + l] = v;
                            }
                    }
                    if (sg.vk) {
#pragma unroll
                        for (int k = 0; k < C::NFK; k++) {  // K_ik: complete
                            double v = 0;
#pragma unroll
                            for (int j = 0; j < C::NFJ; j++)
#pragma unroll
                                for (int l = 0; l < C::NFL; l++) v += A1(j, k, l) * DM(j0 + j, l0 + l);
                            buf[S::OFF_KIK + ci * C::NFK + k] = v;
                        }
#pragma unroll
                        for (int l = 0; l < C::NFL; l++) {  // K_il: complete
                            double v = 0;
#pragma unroll
                            for (int j = 0; j < C::NFJ; j++)
#pragma unroll
                                for (int k = 0; k < C::NFK; k++) v += A1(j, k, l) * DM(j0 + j, k0 + k);
                            buf[S::OFF_KIL + ci * C::NFL + l] = v;
                        }
#pragma unroll
                        for (int j = 0; j < C::NFJ; j++)
#pragma unroll
                            for (int k = 0; k < C::NFK; k++) {  // K_jk: partial over i
                                double v = 0;
#pragma unroll
                                for (int l = 0; l < C::NFL; l++) v += A1(j, k, l) * DM(I, l0 + l);
                                pkjk[j * C::NFK + k] = v;
                            }
#pragma unroll
                        for (int j = 0; j < C::NFJ; j++)
#pragma unroll
                            for (int l = 0; l < C::NFL; l++) {  // K_jl: partial over i
                                double v = 0;
#pragma unroll
                                for (int k = 0; k < C::NFK; k++) v += A1(j, k, l) * DM(I, k0 + k);
                                pkjl[j * C::NFL + l] = v;
                            }
                    }
#undef A1
                } else {
#define A2(k, l) ((double)acc[(k) * C::NFL + (l)])
                    const int I = i0 + ci, J = j0 + cj;
                    double* pjkl = mine;
                    double* pkik = mine + S::NKET;
                    double* pkjk = pkik + C::NFK;
                    double* pkil = pkjk + C::NFK;
                    double* pkjl = pkil + C::NFL;
                    if (sg.vj) {
                        double v = 0;  // J_ij: complete
#pragma unroll
                        for (int k = 0; k < C::NFK; k++)
#pragma unroll
                            for (int l = 0; l < C::NFL; l++) v += A2(k, l) * DM(k0 + k, l0 + l);
                        buf[S::OFF_JIJ + ci * C::NFJ + cj] = v;
                        const double dij = DM(I, J);
#pragma unroll
                        for (int k = 0; k < C::NFK; k++)
#pragma unroll
                            for (int l = 0; l < C::NFL; l++) pjkl[k * C::NFL + l] = A2(k, l) * dij;
                    }
                    if (sg.vk) {
#pragma unroll
                        for (int k = 0; k < C::NFK; k++) {  // K_ik (over j) and K_jk (over i)
                            double vik = 0, vjk = 0;
#pragma unroll
                            for (int l = 0; l < C::NFL; l++) {
                                vik += A2(k, l) * DM(J, l0 + l);
                                vjk += A2(k, l) * DM(I, l0 + l);
                            }
                            pkik[k] = vik;
                            pkjk[k] = vjk;
                        }
#pragma unroll
                        for (int l = 0; l < C::NFL; l++) {  // K_il (over j) and K_jl (over i)
                            double vil = 0, vjl = 0;
#pragma unroll
                            for (int k = 0; k < C::NFK; k++) {
                                vil += A2(k, l) * DM(J, k0 + k);
                                vjl += A2(k, l) * DM(I, k0 + k);
                            }
                            pkil[l] = vil;
                            pkjl[l] = vjl;
                        }
                    }
#undef A2
                }
            }
            __syncthreads();
            if (active) {  // sum the partials of the team into buf
                const double* P0 = part;
                const bool dj = sg.vj != nullptr, dk = sg.vk != nullptr;
                if (dj)
                    for (int b = lane; b < S::NKET; b += T) {
                        double v = 0;
                        for (int t2 = 0; t2 < T; t2++) v += P0[(size_t)t2 * S::PSTRIDE + b];
                        buf[S::OFF_JKL + b] = v;
                    }
                if (dk && C::P == 1) {
                    for (int e = lane; e < C::NFJ * C::NFK; e += T) {
                        double v = 0;
                        for (int t2 = 0; t2 < T; t2++) v += P0[(size_t)t2 * S::PSTRIDE + S::NKET + e];
                        buf[S::OFF_KJK + e] = v;
                    }
                    for (int e = lane; e < C::NFJ * C::NFL; e += T) {
                        double v = 0;
                        for (int t2 = 0; t2 < T; t2++)
                            v += P0[(size_t)t2 * S::PSTRIDE + S::NKET + C::NFJ * C::NFK + e];
                        buf[S::OFF_KJL + e] = v;
                    }
                }
                if (dk && C::P == 2) {
                    // K_ik[i][k] = sum_j, K_jk[j][k] = sum_i, K_il, K_jl likewise
                    for (int e = lane; e < C::NFI * C::NFK; e += T) {
                        int i = e / C::NFK, k = e - i * C::NFK;
                        double v = 0;
                        for (int j = 0; j < C::NFJ; j++)
                            v += P0[(size_t)(i * C::NFJ + j) * S::PSTRIDE + S::NKET + k];
                        buf[S::OFF_KIK + e] = v;
                    }
                    for (int e = lane; e < C::NFJ * C::NFK; e += T) {
                        int j = e / C::NFK, k = e - j * C::NFK;
                        double v = 0;
                        for (int i = 0; i < C::NFI; i++)
                            v += P0[(size_t)(i * C::NFJ + j) * S::PSTRIDE + S::NKET + C::NFK + k];
                        buf[S::OFF_KJK + e] = v;
                    }
                    for (int e = lane; e < C::NFI * C::NFL; e += T) {
                        int i = e / C::NFL, l = e - i * C::NFL;
                        double v = 0;
                        for (int j = 0; j < C::NFJ; j++)
                            v += P0[(size_t)(i * C::NFJ + j) * S::PSTRIDE + S::NKET + 2 * C::NFK + l];
                        buf[S::OFF_KIL + e] = v;
                    }
                    for (int e = lane; e < C::NFJ * C::NFL; e += T) {
                        int j = e / C::NFL, l = e - j * C::NFL;
                        double v = 0;
                        for (int i = 0; i < C::NFI; i++)
                            v += P0[(size_t)(i * C::NFJ + j) * S::PSTRIDE + S::NKET + 2 * C::NFK + C::NFL + l];
                        buf[S::OFF_KJL + e] = v;
                    }
                }
            }
            __syncthreads();
            if (active) {  // flush the team's blocks to global memory
                const int nao = sg.nao;
                const int i0 = q.i0, j0 = q.j0;
                const int k0 = q.k0, l0 = q.l0;
                const size_t moff = (size_t)idm * nao * nao;
                for (int e = lane; e < S::BWORDS_RAW; e += T) {  // not the padding word
                    double v = buf[e];
                    double* V;
                    int a, b;
                    if (e < S::OFF_JKL) { V = sg.vj; a = i0 + e / C::NFJ; b = j0 + e % C::NFJ; }
                    else if (e < S::OFF_KIK) { int x = e - S::OFF_JKL; V = sg.vj; a = k0 + x / C::NFL; b = l0 + x % C::NFL; }
                    else if (e < S::OFF_KIL) { int x = e - S::OFF_KIK; V = sg.vk; a = i0 + x / C::NFK; b = k0 + x % C::NFK; }
                    else if (e < S::OFF_KJK) { int x = e - S::OFF_KIL; V = sg.vk; a = i0 + x / C::NFL; b = l0 + x % C::NFL; }
                    else if (e < S::OFF_KJL) { int x = e - S::OFF_KJK; V = sg.vk; a = j0 + x / C::NFK; b = k0 + x % C::NFK; }
                    else { int x = e - S::OFF_KJL; V = sg.vk; a = j0 + x / C::NFL; b = l0 + x % C::NFL; }
                    if (V) atomicAdd(V + moff + a + (size_t)nao * b, v);
                }
            }
            __syncthreads();
        }
    }
    if (!queue) break;
    }
}
template <class C, typename R>
__global__ void jk_team_kernel(const __grid_constant__ JKSeg sg, const long long* __restrict__ task0) {
    JKOneSeg src{sg, task0};
    jk_team_body<C, R>(src);
}

// ERI-tensor fill with the team kernel's recursion (FP64)
template <class C>
__global__ void jk_team_fill_kernel(const __grid_constant__ JKSeg sg, const long long* __restrict__ task0,
                                    const __grid_constant__ JKFillOut out) {
    JKOneSeg src{sg, task0};
    jk_team_body<C, double>(src, &out);
}

template <class C, typename R>
__global__ void jk_team_kernel_batch(const JKSeg* __restrict__ segs, const long long* __restrict__ segt, int nseg,
                                     unsigned long long* queue, int grab) {
    JKSegTable src{segs, segt, nseg, queue, grab};
    jk_team_body<C, R>(src);
}
#undef DM
