"""Generate the Rys quadrature tables used by the sm_100a ERI kernels.

Rys quadrature (Rys, Dupuis, King, J. Comput. Chem. 4, 154 (1983)) evaluates
the two-electron integrals with an n-point Gauss rule for the measure

    dmu_x(u) = exp(-x u) u^(-1/2) / 2  du,   u = t^2 in [0, 1],

whose moments are the Boys functions F_k(x) = int_0^1 t^(2k) exp(-x t^2) dt.
The n nodes u_i ("roots", the quantity called ``rt`` in the kernels) and
weights w_i satisfy  sum_i w_i u_i^k = F_k(x)  for k = 0 .. 2n-1.

This script computes u_i(x), w_i(x) in 50-digit arithmetic (mpmath):

1. F_0..F_{2n-1} from the convergent series
       F_m(x) = exp(-x) sum_k (2x)^k / ((2m+1)(2m+3)...(2m+2k+1))
   for the top order and downward recursion F_{m-1} = (2x F_m + e^-x)/(2m-1);
2. the three-term recurrence coefficients of the orthogonal polynomials from
   the moments with Gautschi's Chebyshev algorithm (ill conditioned, harmless
   at 50 digits);
3. nodes and weights from the eigen-decomposition of the Jacobi matrix
   (Golub-Welsch).

Each of the 2n functions u_i(x), w_i(x) is stored as a degree-13 Chebyshev
interpolant on intervals of width 2.5 covering 0 <= x < XMAX(n) = 40 + 5n.
Beyond XMAX(n) the measure is indistinguishable from its half-range Hermite
limit (relative error < 1e-15, measured): u_i = s_i^2 / x, w_i = W_i / sqrt(x)
with s_i, W_i the positive nodes and weights of the 2n-point Gauss-Hermite
rule; those 2 x 45 constants are emitted too.

Output: rys_tables.inc (C source, included by the CUDA and C++ sources).
Run:  python -m ccsd_gpu_b200.csrc.gen_rys_tables   (about a minute, 8 cores)
"""
import multiprocessing as mproc
import os
import sys

import mpmath as mp
import numpy as np

NROOTS_MAX = 9
DEGREE = 13            # polynomial degree; DEGREE+1 coefficients per series
WIDTH = 2.5            # interval width in x
DPS = 50


def xmax(n):
    return 40.0 + 5.0 * n


def nintervals(n):
    return int(round(xmax(n) / WIDTH))


def boys_mp(mmax, x):
    x = mp.mpf(x)
    if x == 0:
        return [mp.mpf(1) / (2 * m + 1) for m in range(mmax + 1)]
    ex = mp.exp(-x)
    term = mp.mpf(1) / (2 * mmax + 1)
    s = term
    k = 0
    eps = mp.mpf(10) ** (-mp.mp.dps)
    while True:
        k += 1
        term *= 2 * x / (2 * mmax + 2 * k + 1)
        s += term
        if term < s * eps:
            break
    F = [None] * (mmax + 1)
    F[mmax] = s * ex
    for m in range(mmax, 0, -1):
        F[m - 1] = (2 * x * F[m] + ex) / (2 * m - 1)
    return F


def rys_mp(n, x):
    """Rys nodes (ascending) and weights for n points at argument x."""
    mp.mp.dps = DPS
    mu = boys_mp(2 * n - 1, x)
    sig_prev = [mp.mpf(0)] * (2 * n)
    sig = list(mu)
    alpha = [mu[1] / mu[0]]
    beta = [mu[0]]
    for k in range(1, n):
        new = [mp.mpf(0)] * (2 * n)
        for l in range(k, 2 * n - k):
            new[l] = sig[l + 1] - alpha[k - 1] * sig[l] - beta[k - 1] * sig_prev[l]
        alpha.append(new[k + 1] / new[k] - sig[k] / sig[k - 1])
        beta.append(new[k] / sig[k - 1])
        sig_prev, sig = sig, new
    J = mp.matrix(n, n)
    for i in range(n):
        J[i, i] = alpha[i]
        if i + 1 < n:
            J[i, i + 1] = J[i + 1, i] = mp.sqrt(beta[i + 1])
    E, Q = mp.eigsy(J)
    order = sorted(range(n), key=lambda i: E[i])
    return [E[i] for i in order], [beta[0] * Q[0, i] ** 2 for i in order]


def _node_values(args):
    n, x = args
    r, w = rys_mp(n, x)
    return [float(v) for v in r] + [float(v) for v in w]


def hermite_half(n):
    """Positive nodes s_i (ascending) and weights W_i of the 2n-point Gauss-Hermite rule."""
    mp.mp.dps = DPS
    N = 2 * n
    J = mp.matrix(N, N)
    for k in range(1, N):
        J[k - 1, k] = J[k, k - 1] = mp.sqrt(mp.mpf(k) / 2)
    E, Q = mp.eigsy(J)
    out = sorted((E[i], mp.sqrt(mp.pi) * Q[0, i] ** 2) for i in range(N) if E[i] > 0)
    return [float(s) for s, _ in out], [float(W) for _, W in out]


def chebyshev_coefficients(vals):
    """vals[k] sampled at u_k = cos(pi (k+1/2)/(D+1)); returns c_0..c_D."""
    D = len(vals) - 1
    k = np.arange(D + 1)
    c = np.empty(D + 1)
    for j in range(D + 1):
        c[j] = 2.0 / (D + 1) * np.sum(vals * np.cos(j * np.pi * (k + 0.5) / (D + 1)))
    c[0] *= 0.5
    return c


def build_tables(processes=None):
    k = np.arange(DEGREE + 1)
    unodes = np.cos(np.pi * (k + 0.5) / (DEGREE + 1))
    jobs = []
    for n in range(1, NROOTS_MAX + 1):
        for it in range(nintervals(n)):
            for u in unodes:
                jobs.append((n, it * WIDTH + (u + 1.0) * WIDTH / 2))
    ctx = mproc.get_context("spawn")
    with ctx.Pool(processes) as pool:
        vals = pool.map(_node_values, jobs, chunksize=8)
    # layout: for each n, for each interval, for each series s (u_0..u_{n-1},
    # w_0..w_{n-1}), DEGREE+1 Chebyshev coefficients
    table = []
    offsets = []
    pos = 0
    for n in range(1, NROOTS_MAX + 1):
        offsets.append(len(table))
        nint = nintervals(n)
        block = np.array(vals[pos:pos + nint * (DEGREE + 1)]).reshape(nint, DEGREE + 1, 2 * n)
        pos += nint * (DEGREE + 1)
        for it in range(nint):
            for s in range(2 * n):
                table.extend(chebyshev_coefficients(block[it, :, s]).tolist())
    offsets.append(len(table))
    herm_s, herm_w = [], []
    for n in range(1, NROOTS_MAX + 1):
        s, W = hermite_half(n)
        herm_s.extend(v * v for v in s)
        herm_w.extend(W)
    return table, offsets, herm_s, herm_w


def _fmt(name, vals, ctype="double"):
    lines = ["RYS_TABLE_QUAL %s %s[%d] = {" % (ctype, name, len(vals))]
    for i in range(0, len(vals), 4):
        lines.append("    " + ", ".join(repr(float(v)) if ctype == "double" else str(int(v))
                                        for v in vals[i:i + 4]) + ",")
    lines.append("};")
    return "\n".join(lines)


def write_inc(path, processes=None):
    table, offsets, herm_s2, herm_w = build_tables(processes)
    hdr = [
        "/* Generated by gen_rys_tables.py -- do not edit.",
        " * Rys nodes/weights: degree-%d Chebyshev interpolants on intervals of" % DEGREE,
        " * width %.1f over 0 <= x < 40 + 5 n, n = 1..%d; Hermite limit beyond. */" % (WIDTH, NROOTS_MAX),
        "#ifndef RYS_TABLE_QUAL",
        "#define RYS_TABLE_QUAL static const",
        "#endif",
        "#define RYS_NROOTS_MAX %d" % NROOTS_MAX,
        "#define RYS_DEGREE %d" % DEGREE,
        "#define RYS_WIDTH %.17g" % WIDTH,
        "#define RYS_INV_WIDTH %.17g" % (1.0 / WIDTH),
        "#define RYS_TABLE_SIZE %d" % len(table),
        _fmt("RYS_CHEB_OFFSET", offsets, "int"),
        _fmt("RYS_CHEB", table),
        "/* u_i * x and w_i * sqrt(x) in the large-x limit; entry n(n-1)/2 + i */",
        _fmt("RYS_LARGEX_U", herm_s2),
        _fmt("RYS_LARGEX_W", herm_w),
    ]
    with open(path, "w") as f:
        f.write("\n".join(hdr) + "\n")


if __name__ == "__main__":
    out = sys.argv[1] if len(sys.argv) > 1 else os.path.join(os.path.dirname(__file__), "rys_tables.inc")
    write_inc(out)
    print("wrote", out)
