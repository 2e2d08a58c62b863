// Rys quadrature nodes/weights on the device.
//
// Same quantity as rys_roots_simple (ref: ccsd_gpu/cuda/int2e_ip1_module.py:192-244):
// nodes u_i (= t_i^2) and weights w_i of the n-point Gauss rule for the measure
// exp(-x u) u^(-1/2)/2 du on [0,1], so that sum_i w_i u_i^k = F_k(x).  The tables
// are this project's own (gen_rys_tables.py, 50-digit arithmetic): every node and
// weight is a degree-13 Chebyshev interpolant on width-2.5 intervals up to
// x = 40 + 5n, and the half-range Hermite limit beyond.  Unlike the reference,
// n = 1 and small x use the same tables (no erf formula, no cancellation), and
// every lane evaluates its own quartet's nodes: there is no serial thread-0 step.
#pragma once
#define RYS_TABLE_QUAL __device__ const __align__(16)
#include "rys_tables.inc"
#undef RYS_TABLE_QUAL

namespace cb {

// nodes u[0..n-1] ascending, weights w[0..n-1]; any x (NaN goes to the limit branch,
// the interval index is clamped, so no table access is ever out of range)
static __device__ __noinline__ void rys_roots(int n, double x, double *__restrict__ u,
                                          double *__restrict__ w)
{
    const double xmax = 40.0 + 5.0 * n;
    if (x < xmax) {
        const int nint = 16 + 2 * n;
        int it = (int)(x * RYS_INV_WIDTH);
        it = it < 0 ? 0 : (it >= nint ? nint - 1 : it);
        const double t = (x - it * RYS_WIDTH) * (2.0 * RYS_INV_WIDTH) - 1.0;
        const double t2 = t + t;
        const double *base = RYS_CHEB + RYS_CHEB_OFFSET[n - 1] + it * (2 * n) * (RYS_DEGREE + 1);
        for (int s = 0; s < 2 * n; s++) {
            const double2 *c2 = reinterpret_cast<const double2 *>(base + s * (RYS_DEGREE + 1));
            double c[RYS_DEGREE + 1];
#pragma unroll
            for (int k = 0; k < (RYS_DEGREE + 1) / 2; k++) {
                const double2 v = __ldg(c2 + k);
                c[2 * k] = v.x;
                c[2 * k + 1] = v.y;
            }
            double b1 = 0.0, b2 = 0.0;
#pragma unroll
            for (int k = RYS_DEGREE; k >= 1; k--) {
                const double b0 = fma(t2, b1, c[k] - b2);
                b2 = b1;
                b1 = b0;
            }
            const double v = fma(t, b1, c[0] - b2);
            if (s < n) u[s] = v; else w[s - n] = v;
        }
    } else {
        const int off = n * (n - 1) / 2;
        const double inv = 1.0 / x;
        const double isq = sqrt(inv);
        for (int i = 0; i < n; i++) {
            u[i] = RYS_LARGEX_U[off + i] * inv;
            w[i] = RYS_LARGEX_W[off + i] * isq;
        }
    }
}

// Node r and weight r only (0 <= r < n): the two Chebyshev series run as two
// interleaved, independent Clenshaw chains.  Used where one lane evaluates one
// quadrature point of a primitive quartet, so the lanes of a warp split the n
// points instead of one lane running all 2n series one after the other.
static __device__ __forceinline__ void rys_node(int n, int r, double x, double &u, double &w)
{
    const double xmax = 40.0 + 5.0 * n;
    if (x < xmax) {
        const int nint = 16 + 2 * n;
        int it = (int)(x * RYS_INV_WIDTH);
        it = it < 0 ? 0 : (it >= nint ? nint - 1 : it);
        const double t = (x - it * RYS_WIDTH) * (2.0 * RYS_INV_WIDTH) - 1.0;
        const double t2 = t + t;
        const double *cu = RYS_CHEB + RYS_CHEB_OFFSET[n - 1] + (it * (2 * n) + r) * (RYS_DEGREE + 1);
        const double *cw = cu + n * (RYS_DEGREE + 1);
        double cuv[RYS_DEGREE + 1], cwv[RYS_DEGREE + 1];
#pragma unroll
        for (int k = 0; k < (RYS_DEGREE + 1) / 2; k++) {
            const double2 a = __ldg(reinterpret_cast<const double2 *>(cu) + k);
            const double2 b = __ldg(reinterpret_cast<const double2 *>(cw) + k);
            cuv[2 * k] = a.x;
            cuv[2 * k + 1] = a.y;
            cwv[2 * k] = b.x;
            cwv[2 * k + 1] = b.y;
        }
        double u1 = 0.0, u2 = 0.0, w1 = 0.0, w2 = 0.0;
#pragma unroll
        for (int k = RYS_DEGREE; k >= 1; k--) {
            const double u0 = fma(t2, u1, cuv[k] - u2);
            const double w0 = fma(t2, w1, cwv[k] - w2);
            u2 = u1;
            u1 = u0;
            w2 = w1;
            w1 = w0;
        }
        u = fma(t, u1, cuv[0] - u2);
        w = fma(t, w1, cwv[0] - w2);
    } else {
        const int off = n * (n - 1) / 2;
        const double inv = 1.0 / x;
        u = RYS_LARGEX_U[off + r] * inv;
        w = RYS_LARGEX_W[off + r] * sqrt(inv);
    }
}

}  // namespace cb
