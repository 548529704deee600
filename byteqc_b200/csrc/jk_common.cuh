// Shared device code of the J/K engine: Rys node/weight evaluation, the Rys
// 2D recursion for one (axis, root) unit, Cartesian index helpers and the
// segment descriptors the J/K kernels consume.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// The small per-n metadata is in constant memory of every module; the
// Chebyshev coefficients (about 0.6 MB) are uploaded once per device into
// global memory and reached through a pointer (JKSeg::rys), read with __ldg.
#define RYS_META static __constant__
#include "rys_table.h"

#define JK_LMAX 3      // angular momentum handled by the templated kernels
#define JK_LMAX_ALL 6  // ... and by the generic kernel (jk_generic.cu): up to i
// launcher tables are indexed by the class (li lj | lk ll), base 7
#define JK_CLASS_INDEX(li, lj, lk, ll) ((((li) * 7 + (lj)) * 7 + (lk)) * 7 + (ll))
#define JK_NCLASS 2401

// libcint slots (cuobc/lib/gint/gint.h:29-46)
#define ATM_SLOTS 6
#define PTR_COORD 1
#define BAS_SLOTS 8
#define ATOM_OF 0
#define ANG_OF 1
#define NPRIM_OF 2
#define NCTR_OF 3
#define PTR_EXP 5
#define PTR_COEFF 6

// 2 pi^3 / sqrt(pi): prefactor of the two-electron integrals (the seed of the
// x 2D integrals; cuobc/lib/gint/g2e.c:41)
#define JK_FAC (2.0 * 3.14159265358979323846 * 3.14159265358979323846 * 3.14159265358979323846 / \
                1.77245385090551602730)

// ---------------------------------------------------------------------------
// Rys nodes s_r = t_r^2 and weights w_r at x = rho |P-Q|^2.  The reference
// evaluates the same quantities in the variable u = t^2/(1-t^2)
// (cuobc/lib/gint/rys_roots.cu:1214-2176).
//   n = 1:  w = F0(x), s = F1(x)/F0(x) from the Boys function itself
//           (a Taylor series below x = 0.75, erf/exp above);
//   n > 1:  the generated Chebyshev tables (uniform intervals of width 2 up
//           to rys_xmax[n], Gauss-Hermite limit beyond), evaluated from a
//           copy of the n-root table in shared memory.  Lanes of a warp
//           read the intervals of their own x; the copy's interval stride is
//           odd in doubles so that different intervals start in different
//           banks.
// ---------------------------------------------------------------------------
template <int N>
struct RysS {
    static constexpr int NS = 2 * N;                 // series per interval
    static constexpr int STRIDE = NS * RYS_NC + 1;   // doubles per interval
    static constexpr int NINT = rys_nint_c(N);
    static constexpr int HERM = NINT * STRIDE;       // Gauss-Hermite nodes, then weights
    static constexpr int WORDS = N == 1 ? 0 : HERM + NS;  // doubles in shared memory
    static constexpr double XMAX = rys_xmax_c(N);
};

// block-cooperative copy of the n-root table into shared memory (layout
// [interval][k][series], series f < N nodes, f >= N weights)
template <int N>
__device__ __forceinline__ void rys_table_to_smem(const double* __restrict__ g, double* __restrict__ tab) {
    using S = RysS<N>;
    if (N == 1) return;
    const double* src = g + rys_off_c(N);
    for (int e = threadIdx.x; e < S::NINT * S::NS * RYS_NC; e += blockDim.x) {
        int m = e / (S::NS * RYS_NC);
        int rem = e - m * (S::NS * RYS_NC);
        int f = rem / RYS_NC, k = rem - f * RYS_NC;
        tab[m * S::STRIDE + k * S::NS + f] = __ldg(src + e);
    }
    for (int r = threadIdx.x; r < N; r += blockDim.x) {
        tab[S::HERM + r] = rys_herm_r[N * (N - 1) / 2 + r];
        tab[S::HERM + N + r] = rys_herm_w[N * (N - 1) / 2 + r];
    }
}

// F0 and F1 of the Boys function
__device__ __forceinline__ void boys01(double x, double& f0, double& f1) {
    if (x < 0.75) {
        // F_m(x) = sum_k (-x)^k / (k! (2m + 2k + 1)), 19 terms (< 1e-18 at 0.75)
        double a0 = 0., a1 = 0., fk = 1.;
        double c0[19], c1[19];
#pragma unroll
        for (int k = 0; k < 19; k++) {
            if (k) fk *= k;
            c0[k] = ((k & 1) ? -1. : 1.) / (fk * (2 * k + 1));
            c1[k] = ((k & 1) ? -1. : 1.) / (fk * (2 * k + 3));
        }
#pragma unroll
        for (int k = 18; k >= 0; k--) {
            a0 = fma(a0, x, c0[k]);
            a1 = fma(a1, x, c1[k]);
        }
        f0 = a0;
        f1 = a1;
    } else if (x < 40.) {
        const double rx = rsqrt(x), sx = x * rx;        // 1/sqrt(x), sqrt(x)
        f0 = 0.88622692545275801365 * erf(sx) * rx;     // sqrt(pi)/2 erf(sqrt x)/sqrt x
        f1 = (f0 - exp(-x)) * (0.5 * rx * rx);         // (F0 - e^-x) / (2x)
    } else {
        // asymptotic: erfc(sqrt 40) < 1e-18 and e^-40 / F0 < 3e-17, below the
        // double rounding of the terms kept
        const double rx = rsqrt(x);
        f0 = 0.88622692545275801365 * rx;
        f1 = f0 * (0.5 * rx * rx);
    }
}

// Rys node r at x with the root count N known at run time (the layout and
// evaluation of rys_root<N>)
__device__ __forceinline__ void rys_root_rt(const double* __restrict__ rys, int N, double x, int r, double& s, double& w) {
    if (N == 1) {
        double f0, f1;
        boys01(x, f0, f1);
        w = f0;
        s = f1 / f0;
        return;
    }
    if (x >= rys_xmax_c(N)) {
        const int b = N * (N - 1) / 2 + r;
        const double rx = 1. / x;
        s = rys_herm_r[b] * rx;
        w = rys_herm_w[b] * sqrt(rx);
        return;
    }
    const int m = (int)(x * 0.5);
    const double t = x - (2 * m + 1), tt = t + t;
    const double* c = rys + rys_off_c(N) + (size_t)(m * 2 * N) * RYS_NC;
    const double* cs = c + r * RYS_NC;
    const double* cw = c + (N + r) * RYS_NC;
    double b1 = 0., b2 = 0., v1 = 0., v2 = 0.;
    for (int k = RYS_NC - 1; k >= 1; k--) {
        double b0 = fma(tt, b1, __ldg(cs + k) - b2);
        b2 = b1;
        b1 = b0;
        b0 = fma(tt, v1, __ldg(cw + k) - v2);
        v2 = v1;
        v1 = b0;
    }
    s = fma(t, b1, __ldg(cs) - b2);
    w = fma(t, v1, __ldg(cw) - v2);
}

// all N roots at x from the shared-memory table
template <int N>
__device__ __forceinline__ void rys_roots_all(const double* __restrict__ tab, double x, double* s, double* w) {
    using S = RysS<N>;
    if (N == 1) {
        double f0, f1;
        boys01(x, f0, f1);
        w[0] = f0;
        s[0] = f1 / f0;
        return;
    }
    if (x >= S::XMAX) {
        double rx = 1. / x, srx = sqrt(rx);
#pragma unroll
        for (int r = 0; r < N; r++) {
            s[r] = tab[S::HERM + r] * rx;
            w[r] = tab[S::HERM + N + r] * srx;
        }
        return;
    }
    int m = (int)(x * 0.5);
    double t = x - (2 * m + 1), t2 = t + t;
    const double* c = tab + m * S::STRIDE;
    double b1[S::NS], b2[S::NS];
#pragma unroll
    for (int f = 0; f < S::NS; f++) b1[f] = b2[f] = 0.;
#pragma unroll
    for (int k = RYS_NC - 1; k >= 1; k--) {
#pragma unroll
        for (int f = 0; f < S::NS; f++) {
            double b0 = fma(t2, b1[f], c[k * S::NS + f] - b2[f]);
            b2[f] = b1[f];
            b1[f] = b0;
        }
    }
#pragma unroll
    for (int r = 0; r < N; r++) {
        s[r] = fma(t, b1[r], c[r] - b2[r]);
        w[r] = fma(t, b1[N + r], c[N + r] - b2[N + r]);
    }
}

// root r only (runtime r) from the shared-memory table
template <int N>
__device__ __forceinline__ void rys_root_one(const double* __restrict__ tab, double x, int r, double& s, double& w) {
    using S = RysS<N>;
    if (N == 1) {
        double f0, f1;
        boys01(x, f0, f1);
        w = f0;
        s = f1 / f0;
        return;
    }
    if (x >= S::XMAX) {
        double rx = 1. / x;
        s = tab[S::HERM + r] * rx;
        w = tab[S::HERM + N + r] * sqrt(rx);
        return;
    }
    int m = (int)(x * 0.5);
    double t = x - (2 * m + 1), t2 = t + t;
    const double* c = tab + m * S::STRIDE;
    double bs1 = 0., bs2 = 0., bw1 = 0., bw2 = 0.;
#pragma unroll
    for (int k = RYS_NC - 1; k >= 1; k--) {
        double b0 = fma(t2, bs1, c[k * S::NS + r] - bs2);
        bs2 = bs1;
        bs1 = b0;
        b0 = fma(t2, bw1, c[k * S::NS + N + r] - bw2);
        bw2 = bw1;
        bw1 = b0;
    }
    s = fma(t, bs1, c[r] - bs2);
    w = fma(t, bw1, c[N + r] - bw2);
}

// root r straight from the global table (setup kernels)
template <int N>
__device__ __forceinline__ void rys_root(const double* __restrict__ rys_coef, double x, int r, double& s,
                                         double& w) {
    if (N == 1) {
        double f0, f1;
        boys01(x, f0, f1);
        w = f0;
        s = f1 / f0;
        return;
    }
    if (x >= rys_xmax_c(N)) {
        int b = N * (N - 1) / 2 + r;
        double rx = 1. / x;
        s = rys_herm_r[b] * rx;
        w = rys_herm_w[b] * sqrt(rx);
        return;
    }
    int m = (int)(x * 0.5);
    double t = x - (2 * m + 1);
    const double* c = rys_coef + rys_off_c(N) + (m * 2 * N) * RYS_NC;
    double b1 = 0., b2 = 0., v1 = 0., v2 = 0., tt = t + t;
    const double* cs = c + r * RYS_NC;
    const double* cw = c + (N + r) * RYS_NC;
#pragma unroll
    for (int k = RYS_NC - 1; k >= 1; k--) {
        double b0 = fma(tt, b1, __ldg(cs + k) - b2);
        b2 = b1;
        b1 = b0;
        b0 = fma(tt, v1, __ldg(cw + k) - v2);
        v2 = v1;
        v1 = b0;
    }
    s = fma(t, b1, __ldg(cs) - b2);
    w = fma(t, v1, __ldg(cw) - v2);
}

// ---------------------------------------------------------------------------
// Single-precision nodes and weights for the FP32 quartets of the mixed mode
// at low order (n <= JK_F32_ROOTS): the Boys function in float for n = 1, the
// same Chebyshev tables rounded to float for n = 2, 3.  Higher orders keep
// the double evaluation above.  Same shared-memory layout as the double copy
// (the stride is odd in floats too).
// ---------------------------------------------------------------------------
#define JK_F32_ROOTS 3

template <int N>
__device__ __forceinline__ void rys_table_to_smem_f(const double* __restrict__ g, float* __restrict__ tab) {
    using S = RysS<N>;
    if (N == 1) return;
    const double* src = g + rys_off_c(N);
    for (int e = threadIdx.x; e < S::NINT * S::NS * RYS_NC; e += blockDim.x) {
        int m = e / (S::NS * RYS_NC);
        int rem = e - m * (S::NS * RYS_NC);
        int f = rem / RYS_NC, k = rem - f * RYS_NC;
        tab[m * S::STRIDE + k * S::NS + f] = (float)__ldg(src + e);
    }
    for (int r = threadIdx.x; r < N; r += blockDim.x) {
        tab[S::HERM + r] = (float)rys_herm_r[N * (N - 1) / 2 + r];
        tab[S::HERM + N + r] = (float)rys_herm_w[N * (N - 1) / 2 + r];
    }
}

// F0 and F1 in float: the series below x = 0.75 (12 terms, truncation below
// 1e-10), erf/exp above
__device__ __forceinline__ void boys01_f(float x, float& f0, float& f1) {
    if (x < 0.75f) {
        float a0 = 0.f, a1 = 0.f;
        double fk = 1.;
        float c0[12], c1[12];
#pragma unroll
        for (int k = 0; k < 12; k++) {
            if (k) fk *= k;
            c0[k] = (float)(((k & 1) ? -1. : 1.) / (fk * (2 * k + 1)));
            c1[k] = (float)(((k & 1) ? -1. : 1.) / (fk * (2 * k + 3)));
        }
#pragma unroll
        for (int k = 11; k >= 0; k--) {
            a0 = fmaf(a0, x, c0[k]);
            a1 = fmaf(a1, x, c1[k]);
        }
        f0 = a0;
        f1 = a1;
    } else {
        float rsx = rsqrtf(x);
        f0 = 0.886226925f * erff(x * rsx) * rsx;  // sqrt(pi)/2 erf(sqrt x)/sqrt x
        f1 = (f0 - expf(-x)) * (0.5f * rsx * rsx);
    }
}

template <int N>
__device__ __forceinline__ void rys_roots_all_f(const float* __restrict__ tab, float x, float* s, float* w) {
    using S = RysS<N>;
    if (N == 1) {
        float f0, f1;
        boys01_f(x, f0, f1);
        w[0] = f0;
        s[0] = __fdividef(f1, f0);
        return;
    }
    if (x >= (float)S::XMAX) {
        float srx = rsqrtf(x), rx = srx * srx;
#pragma unroll
        for (int r = 0; r < N; r++) {
            s[r] = tab[S::HERM + r] * rx;
            w[r] = tab[S::HERM + N + r] * srx;
        }
        return;
    }
    int m = (int)(x * 0.5f);
    float t = x - (float)(2 * m + 1), t2 = t + t;
    const float* c = tab + m * S::STRIDE;
    float b1[S::NS], b2[S::NS];
#pragma unroll
    for (int f = 0; f < S::NS; f++) b1[f] = b2[f] = 0.f;
#pragma unroll
    for (int k = RYS_NC - 1; k >= 1; k--) {
#pragma unroll
        for (int f = 0; f < S::NS; f++) {
            float b0 = fmaf(t2, b1[f], c[k * S::NS + f] - b2[f]);
            b2[f] = b1[f];
            b1[f] = b0;
        }
    }
#pragma unroll
    for (int r = 0; r < N; r++) {
        s[r] = fmaf(t, b1[r], c[r] - b2[r]);
        w[r] = fmaf(t, b1[N + r], c[N + r] - b2[N + r]);
    }
}

// root r only (runtime r), single precision, from the float table copy
template <int N>
__device__ __forceinline__ void rys_root_one_f(const float* __restrict__ tab, float x, int r, float& s, float& w) {
    using S = RysS<N>;
    if (N == 1) {
        float f0, f1;
        boys01_f(x, f0, f1);
        w = f0;
        s = __fdividef(f1, f0);
        return;
    }
    if (x >= (float)S::XMAX) {
        const float srx = rsqrtf(x);
        s = tab[S::HERM + r] * srx * srx;
        w = tab[S::HERM + N + r] * srx;
        return;
    }
    const int m = (int)(x * 0.5f);
    const float t = x - (float)(2 * m + 1), t2 = t + t;
    const float* c = tab + m * S::STRIDE;
    float bs1 = 0.f, bs2 = 0.f, bw1 = 0.f, bw2 = 0.f;
#pragma unroll
    for (int k = RYS_NC - 1; k >= 1; k--) {
        float b0 = fmaf(t2, bs1, c[k * S::NS + r] - bs2);
        bs2 = bs1;
        bs1 = b0;
        b0 = fmaf(t2, bw1, c[k * S::NS + N + r] - bw2);
        bw2 = bw1;
        bw1 = b0;
    }
    s = fmaf(t, bs1, c[r] - bs2);
    w = fmaf(t, bw1, c[N + r] - bw2);
}

// ---------------------------------------------------------------------------
// Compile-time class description for (li lj | lk ll), li >= lj, lk >= ll.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// Exponents of Cartesian component c of angular momentum l in libcint order
// (lx descending, then ly descending).  With u = l - lx, the components with
// x exponent above lx number u(u+1)/2, so u is the triangular root of c and
// lz = c - u(u+1)/2.  Loop-free so that unrolled loops fold them to constants.
__host__ __device__ constexpr int cart_u(int c) {
    return c < 1 ? 0 : c < 3 ? 1 : c < 6 ? 2 : c < 10 ? 3 : c < 15 ? 4 : c < 21 ? 5 : 6;
}
__host__ __device__ constexpr int cart_lz(int l, int c) { return c - cart_u(c) * (cart_u(c) + 1) / 2; }
__host__ __device__ constexpr int cart_lx(int l, int c) { return l - cart_u(c); }
__host__ __device__ constexpr int cart_ly(int l, int c) { return cart_u(c) - cart_lz(l, c); }

template <int LI_, int LJ_, int LK_, int LL_>
struct JKClass {
    static constexpr int LI = LI_, LJ = LJ_, LK = LK_, LL = LL_;
    static constexpr int NFI = ncart(LI), NFJ = ncart(LJ), NFK = ncart(LK), NFL = ncart(LL);
    static constexpr int NF = NFI * NFJ * NFK * NFL;
    static constexpr int NROOTS = (LI + LJ + LK + LL) / 2 + 1;
    static constexpr int NM = LI + LJ, MM = LK + LL;
    // strides of the per-unit 2D integral block I[i][j][k][l]
    static constexpr int SL = 1, SK = LL + 1, SJ = (LK + 1) * (LL + 1), SI = (LJ + 1) * (LK + 1) * (LL + 1);
    static constexpr int GS = (LI + 1) * SI;
    // ownership: P leading centres are owned by a thread of the team; the
    // remaining Cartesian components are accumulated in registers
    // One thread per quartet (P = 0) when one root's 2D blocks and the
    // accumulators of GI bra components fit in registers: in one pass if all
    // components fit (W <= 64 doubles), else in NPASS <= 4 passes over the
    // primitives with GI bra components each (<= 80 doubles live).  Larger
    // classes use a team per quartet (P = 1: owned i; P = 2: owned i and j).
    static constexpr int EI = NFJ * NFK * NFL;  // components per bra index
    static constexpr int GI1 = (80 - 3 * GS) / EI;
    static constexpr int GI = (NF + 3 * GS <= 64) ? NFI : (3 * GS <= 48 && GI1 >= 1 ? GI1 : 0);
    static constexpr int NPASS = GI ? (NFI + GI - 1) / GI : 0;
    static constexpr bool THREAD = GI > 0 && NPASS <= 4;
    static constexpr int W = (THREAD ? (GI < NFI ? GI : NFI) * EI : NF) + 3 * GS;
    static constexpr int P = THREAD ? 0 : ((NF / NFI <= 64) ? 1 : 2);
    static constexpr int T = P == 0 ? 1 : (P == 1 ? NFI : NFI * NFJ);
    static constexpr int NACC = NF / T;
    // resident 128-thread blocks asked of the register allocator (thread kernel)
    static constexpr int MINB = W <= 24 ? 4 : (W <= 40 ? 3 : 2);
};

// ---------------------------------------------------------------------------
// One Rys 2D block (one axis, one root).  VRR builds G[n][m] on the bra
// centre i and ket centre k:
//   G[n+1][0]   = c00 G[n][0] + n b10 G[n-1][0]
//   G[n][m+1]   = c0p G[n][m] + m b01 G[n][m-1] + n b00 G[n-1][m]
// then the horizontal transfers (a, j+1) = (a+1, j) + (Ri - Rj)(a, j) and
// (c, l+1) = (c+1, l) + (Rk - Rl)(c, l).  Same recursion as the reference's
// GINTg0_2e_2d4d (cuobc/lib/gvhf/g2e.cu:66-166), written here as explicit
// register arrays.  Output: I[i*XSI + j*XSJ + k*(LL+1) + l], by default the
// packed layout I[((i*(LJ+1)+j)*(LK+1)+k)*(LL+1)+l].
// ---------------------------------------------------------------------------
template <typename R, class C, int XSI = C::SI, int XSJ = C::SJ, typename OutT>
__device__ __forceinline__ void rys_2d(R seed, R c00, R c0p, R b10, R b01, R b00, R dij, R dkl,
                                       OutT* __restrict__ I) {
    constexpr int NM = C::NM, MM = C::MM;
    R G[NM + 1][MM + 1];
    G[0][0] = seed;
#pragma unroll
    for (int n = 0; n < NM; n++) G[n + 1][0] = c00 * G[n][0] + (n ? R(n) * b10 * G[n > 0 ? n - 1 : 0][0] : R(0));
#pragma unroll
    for (int m = 0; m < MM; m++) {
#pragma unroll
        for (int n = 0; n <= NM; n++) {
            R v = c0p * G[n][m];
            if (m) v += R(m) * b01 * G[n][m > 0 ? m - 1 : 0];
            if (n) v += R(n) * b00 * G[n > 0 ? n - 1 : 0][m];
            G[n][m + 1] = v;
        }
    }
    // bra transfer: H[i][j][m]
    R H[C::LI + 1][C::LJ + 1][MM + 1];
#pragma unroll
    for (int m = 0; m <= MM; m++) {
        R A[NM + 1];
#pragma unroll
        for (int a = 0; a <= NM; a++) A[a] = G[a][m];
#pragma unroll
        for (int i = 0; i <= C::LI; i++) H[i][0][m] = A[i];
#pragma unroll
        for (int j = 1; j <= C::LJ; j++) {
#pragma unroll
            for (int a = 0; a + j <= NM; a++) A[a] = A[a + 1] + dij * A[a];
#pragma unroll
            for (int i = 0; i <= C::LI; i++) H[i][j][m] = A[i];
        }
    }
    // ket transfer
#pragma unroll
    for (int i = 0; i <= C::LI; i++)
#pragma unroll
        for (int j = 0; j <= C::LJ; j++) {
            R B[MM + 1];
#pragma unroll
            for (int c = 0; c <= MM; c++) B[c] = H[i][j][c];
#pragma unroll
            for (int k = 0; k <= C::LK; k++) I[i * XSI + j * XSJ + k * C::SK] = B[k];
#pragma unroll
            for (int l = 1; l <= C::LL; l++) {
#pragma unroll
                for (int c = 0; c + l <= MM; c++) B[c] = B[c + 1] + dkl * B[c];
#pragma unroll
                for (int k = 0; k <= C::LK; k++) I[i * XSI + j * XSJ + k * C::SK + l] = B[k];
            }
        }
}

// ---------------------------------------------------------------------------
// Segment: one (molecule, class quartet) piece of work.  Tasks of a segment
// are the screened contracted shell quartets (ij, kl), enumerated row by row:
// row ij holds kl = 0 .. nkl(ij)-1 and qoff is the exclusive prefix of nkl.
// ---------------------------------------------------------------------------
struct JKSeg {
    const double* rys;      // Rys coefficient table (device)
    const long long* qoff;  // n_ij + 1 entries (device)
    const int* kl_base;     // first kl column of each row (FP32 part of the mixed mode), or null
    int n_ij;
    int pair_ij0, pair_kl0;  // first pair of each class in the pair arrays
    int prim_ij0, prim_kl0;  // first primitive pair of each class
    int nprim_ij, nprim_kl;
    // primitive pairs are stored primitive-major within a class: primitive
    // k of pair r at prim0 + k*pst + r (pst = pairs in the class), so the
    // lanes of a warp (consecutive kl pairs) load them coalesced
    int pst_ij, pst_kl;
    int nao, n_dm;
    const int* pair2bra;
    const int* pair2ket;
    const double* a12;
    const double* ia12;  // 1 / a12
    const double* e12;
    const double* x12;
    const double* y12;
    const double* z12;
    // FP32 copy of the primitive pairs for the FP32 quartets of the mixed
    // mode, SoA of npf floats each: a12 | 1/a12 | e12/a12 | P - R_bra (x, y, z)
    const float* pf;
    long long npf;
    // pair geometry, indexed by pair (stride npt): the centres of the pair's
    // two shells (SoA x_a y_a z_a x_b y_b z_b) and their first AOs (SoA
    // ao_a ao_b); one dependent load per quartet side instead of two, and
    // coalesced on the ket side (consecutive lanes hold consecutive pairs)
    const double* pgeo;
    const int* pao;
    int npt;
    // per pair: its leading primitive pairs that pass the exponent cutoff
    // (the thread kernels loop over those only), or null
    const int* pnp;
    const double* bas_x;  // shell centres, SoA x[nbas], y[nbas], z[nbas]
    int nbas;
    const int* ao_loc;
    const double* dm;
    double* vj;
    double* vk;
    // Pair-packed J side (jk_build): the density blocks of the pairs of the
    // two classes, component-major (element c of pair p of a class at
    // c * np + p), and accumulators of the same layout for the J
    // contributions, added to vj after the launches.  Null: the kernels
    // gather D and add J straight into vj.
    const double* dp_ij;
    const double* dp_kl;
    double* jp_ij;
    double* jp_kl;
    int np_ij, np_kl;        // pairs of each class (component stride)
    long long pk_stride;     // packed elements per density
    int ls[4];               // angular momenta of the class (read by the generic kernel)
};

// launchers of one class: a single segment (by value) or a segment table
typedef cudaError_t (*jk_launch_fn)(const JKSeg& seg, const long long* task0, long long max_tasks, int nsm,
                                    cudaStream_t st);
// Launch shape of one batched class launch (the knobs of the batch's
// autotuner).  queue == nullptr: the tasks are split into equal contiguous
// chunks over a grid sized by the unscreened task count.  Otherwise the
// persistent mode: the grid is grid_mul x the kernel's resident blocks per
// SM x the SMs, and the warps (thread kernels), teams (team kernels) or
// blocks (generic kernel) take `grab` tasks at a time from the device
// counter *queue, which the caller zeroes before the launch.
struct JKBatchCfg {
    unsigned long long* queue;
    int grab;
    int grid_mul;
};
typedef cudaError_t (*jk_launch_batch_fn)(const JKSeg* segs, const long long* segt, int nseg, long long max_tasks,
                                          int nsm, const JKBatchCfg& cfg, cudaStream_t st);

