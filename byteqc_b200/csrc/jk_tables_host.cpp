// Host-side evaluation of the generated Rys tables (the same series the
// device evaluates in jk_common.cuh), exported for checking the tables.
#include <math.h>

#define RYS_META static const
#define RYS_WANT_COEF
#include "rys_table.h"

#include "../../include/byteqc_jk.h"

static double cheb(const double* c, double t) {
    double b1 = 0., b2 = 0., t2 = t + t;
    for (int k = RYS_NC - 1; k >= 1; k--) {
        double b0 = fma(t2, b1, c[k] - b2);
        b2 = b1;
        b1 = b0;
    }
    return fma(t, b1, c[0] - b2);
}

extern "C" int jk_rys_roots_host(int n, double x, double* s, double* w) {
    if (n < 1 || n > RYS_NMAX || !(x >= 0) || !s || !w) return JK_ERR_ARG;
    if (x >= rys_xmax[n]) {
        int b = n * (n - 1) / 2;
        double rx = 1. / x;
        for (int r = 0; r < n; r++) {
            s[r] = rys_herm_r[b + r] * rx;
            w[r] = rys_herm_w[b + r] * sqrt(rx);
        }
        return JK_OK;
    }
    double h = rys_h[n];
    int m = (int)(x / h);
    double t = (x - (m + 0.5) * h) / (0.5 * h);
    const double* c = rys_coef + rys_off[n] + (m * 2 * n) * RYS_NC;
    for (int r = 0; r < n; r++) {
        s[r] = cheb(c + r * RYS_NC, t);
        w[r] = cheb(c + (n + r) * RYS_NC, t);
    }
    return JK_OK;
}

extern "C" int jk_rys_table_uniform(void) {
    for (int n = 1; n <= RYS_NMAX; n++)
        if (rys_h[n] != 2.0) return 0;
    return 1;
}

// the coefficient table, uploaded to each device by the engine
extern "C" const double* jk_rys_coef_host(long long* count) {
    if (count) *count = RYS_TOTAL;
    return rys_coef;
}
