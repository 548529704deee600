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

#define JK_LMAX 3  // angular momentum handled by the templated kernels

// 2 pi^3 / sqrt(pi): prefactor of the two-electron integrals (the seed of the
// x 2D integrals; cuobc/lib/gint/g2e.c:41)
#define JK_FAC (2.0 * 3.14159265358979323846 * 3.14159265358979323846 * 3.14159265358979323846 / \
                1.77245385090551602730)

// ---------------------------------------------------------------------------
// Rys nodes s_r = t_r^2 and weights w_r at x = rho |P-Q|^2 from the generated
// Chebyshev tables (uniform intervals of width rys_h[n] up to rys_xmax[n],
// Gauss-Hermite limit beyond).  The reference evaluates the same quantities
// in the variable u = t^2/(1-t^2) (cuobc/lib/gint/rys_roots.cu:1214-2176).
// ---------------------------------------------------------------------------
__device__ __forceinline__ double rys_cheb(const double* __restrict__ c, double t) {
    double b1 = 0., b2 = 0., t2 = t + t;
#pragma unroll
    for (int k = RYS_NC - 1; k >= 1; k--) {
        double b0 = fma(t2, b1, __ldg(c + k) - b2);
        b2 = b1;
        b1 = b0;
    }
    return fma(t, b1, __ldg(c) - b2);
}

template <int N>
__device__ __forceinline__ void rys_root(const double* __restrict__ rys_coef, double x, int r, double& s,
                                         double& w) {
    if (x >= rys_xmax[N]) {
        int b = N * (N - 1) / 2 + r;
        double rx = 1. / x;
        s = rys_herm_r[b] * rx;
        w = rys_herm_w[b] * sqrt(rx);
        return;
    }
    // rys_h is 2 for every n (checked by the host at load time)
    int m = (int)(x * 0.5);
    double t = x - (2 * m + 1);
    const double* c = rys_coef + rys_off[N] + (m * 2 * N) * RYS_NC;
    s = rys_cheb(c + r * RYS_NC, t);
    w = rys_cheb(c + (N + r) * RYS_NC, t);
}

// ---------------------------------------------------------------------------
// Compile-time class description for (li lj | lk ll), li >= lj, lk >= ll.
// ---------------------------------------------------------------------------
__host__ __device__ constexpr int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// x and y exponents of Cartesian component c of angular momentum l in libcint
// order (lx descending, then ly descending)
__host__ __device__ constexpr int cart_lx(int l, int c) {
    int lx = l;
    while (c > l - lx) {
        c -= l - lx + 1;
        lx--;
    }
    return lx;
}
__host__ __device__ constexpr int cart_ly(int l, int c) {
    int lx = l;
    while (c > l - lx) {
        c -= l - lx + 1;
        lx--;
    }
    return l - lx - c;
}
__host__ __device__ constexpr int cart_lz(int l, int c) { return l - cart_lx(l, c) - cart_ly(l, c); }

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
    static constexpr int P = (NF <= 64) ? 0 : ((NF / NFI <= 64) ? 1 : 2);
    static constexpr int T = P == 0 ? 1 : (P == 1 ? NFI : NFI * NFJ);
    static constexpr int NACC = NF / T;
};

// ---------------------------------------------------------------------------
// One Rys 2D block (one axis, one root).  VRR builds G[n][m] on the bra
// centre i and ket centre k:
//   G[n+1][0]   = c00 G[n][0] + n b10 G[n-1][0]
//   G[n][m+1]   = c0p G[n][m] + m b01 G[n][m-1] + n b00 G[n-1][m]
// then the horizontal transfers (a, j+1) = (a+1, j) + (Ri - Rj)(a, j) and
// (c, l+1) = (c+1, l) + (Rk - Rl)(c, l).  Same recursion as the reference's
// GINTg0_2e_2d4d (cuobc/lib/gvhf/g2e.cu:66-166), written here as explicit
// register arrays.  Output: I[((i*(LJ+1)+j)*(LK+1)+k)*(LL+1)+l].
// ---------------------------------------------------------------------------
template <typename R, class C, typename OutT>
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
            for (int k = 0; k <= C::LK; k++) I[i * C::SI + j * C::SJ + k * C::SK] = B[k];
#pragma unroll
            for (int l = 1; l <= C::LL; l++) {
#pragma unroll
                for (int c = 0; c + l <= MM; c++) B[c] = B[c + 1] + dkl * B[c];
#pragma unroll
                for (int k = 0; k <= C::LK; k++) I[i * C::SI + j * C::SJ + k * C::SK + l] = B[k];
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
    int n_ij;
    int pair_ij0, pair_kl0;  // first pair of each class in the pair arrays
    int prim_ij0, prim_kl0;  // first primitive pair of each class
    int nprim_ij, nprim_kl;
    int nao, n_dm;
    const int* pair2bra;
    const int* pair2ket;
    const double* a12;
    const double* e12;
    const double* x12;
    const double* y12;
    const double* z12;
    const double* bas_x;  // shell centres, SoA x[nbas], y[nbas], z[nbas]
    int nbas;
    const int* ao_loc;
    const double* dm;
    double* vj;
    double* vk;
};
