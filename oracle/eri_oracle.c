/*
 * ORACLE -- test infrastructure only.  Nothing in ccsd_gpu_b200/ links this.
 *
 * CPU restatement of the reference's two-electron integral path:
 *   - Rys roots/weights          (ref: ccsd_gpu/cuda/int2e_ip1_module.py:192-244)
 *   - fill_int2e_kernel          (ref: ccsd_gpu/cuda/int2e_module.py:130-463)
 *   - fill_int2e_ip1_kernel      (ref: ccsd_gpu/cuda/int2e_ip1_module.py:273-667)
 *   - s2kl output layout         (ref: ccsd_gpu/cuda/int2e_gpu.py:186-215,
 *                                      ccsd_gpu/cuda/int2e_ip1_gpu.py:296-326)
 *
 * The Rys nodes/weights here do NOT use the kernels' Chebyshev tables: they
 * are recomputed per call by the discretised Stieltjes procedure (Gautschi,
 * "Orthogonal polynomials: computation and approximation", 2004, sec. 2.2.3)
 * in long double on a 240-point Gauss-Legendre discretisation of
 * int_0^1 f(t^2) exp(-x t^2) dt, followed by an implicit-QL eigen-solve of
 * the Jacobi matrix (Golub-Welsch).  For x above 40 + 5n the half-range
 * Gauss-Hermite limit is used (relative error < 1e-15 there).
 *
 * Integral recurrences (Rys, Dupuis & King, J. Comput. Chem. 4, 154 (1983)):
 *   I(n+1,0)   = C00  I(n,0) + n B10 I(n-1,0)
 *   I(n,m+1)   = C00' I(n,m) + m B01 I(n,m-1) + n B00 I(n-1,m)
 *   I(i,j+1)   = I(i+1,j) + (A-B) I(i,j)         (same for k,l with C-D)
 * with B00 = u/2(p+q), B10 = (1 - u q/(p+q))/2p, B01 = (1 - u p/(p+q))/2q,
 * C00 = (P-A) - u q/(p+q) (P-Q), C00' = (Q-C) + u p/(p+q) (P-Q).
 *
 * Conventions follow PySCF/libcint: shells described by _atm/_bas/_env,
 * coefficients in env already carry the radial normalisation, s and p
 * Cartesian functions carry the angular factor 1/(2 sqrt(pi)) and
 * sqrt(3)/(2 sqrt(pi)); Cartesian components in lexicographic order
 * (xx, xy, xz, yy, yz, zz, ...).  int2e_ip1 is (d/dr_1 i j|kl) =
 *   l_x I(i-1) - 2 a_i I(i+1).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define ATM_SLOTS 6
#define PTR_COORD 1
#define BAS_SLOTS 8
#define ATOM_OF 0
#define ANG_OF 1
#define NPRIM_OF 2
#define NCTR_OF 3
#define PTR_EXP 5
#define PTR_COEFF 6

#define NGL 240
#define NMAX 9
#define LMAX 4

static long double gl_t[NGL], gl_v[NGL];
static int gl_ready = 0;

/* Gauss-Legendre nodes on [0,1] by Newton iteration on P_N. */
static void gl_init(void)
{
    if (gl_ready) return;
#pragma omp critical(oracle_gl_init)
    {
    if (!gl_ready) {
    const int N = NGL;
    for (int i = 0; i < N; i++) {
        long double z = cosl(3.14159265358979323846264338327950288L * (i + 0.75L) / (N + 0.5L));
        long double pp = 0;
        for (int it = 0; it < 100; it++) {
            long double p1 = 1, p2 = 0;
            for (int j = 1; j <= N; j++) {
                long double p3 = p2;
                p2 = p1;
                p1 = ((2 * j - 1) * z * p2 - (j - 1) * p3) / j;
            }
            pp = N * (z * p1 - p2) / (z * z - 1);
            long double dz = p1 / pp;
            z -= dz;
            if (fabsl(dz) < 1e-19L) break;
        }
        gl_t[i] = 0.5L * (1 - z);
        gl_v[i] = 1.0L / ((1 - z * z) * pp * pp);   /* = w_GL / 2 */
    }
    gl_ready = 1;
    }
    }
}

/* Symmetric tridiagonal eigenproblem, implicit QL (diag d, offdiag e[1..n-1]);
 * z returns the first row of the eigenvector matrix. */
static void tqli(long double *d, long double *e, int n, long double *z)
{
    for (int i = 0; i < n; i++) z[i] = (i == 0);
    for (int i = 1; i < n; i++) e[i - 1] = e[i];
    e[n - 1] = 0;
    for (int l = 0; l < n; l++) {
        int iter = 0, m;
        do {
            for (m = l; m < n - 1; m++) {
                long double dd = fabsl(d[m]) + fabsl(d[m + 1]);
                if (fabsl(e[m]) <= 1e-21L * dd) break;
            }
            if (m != l) {
                if (iter++ == 200) break;
                long double g = (d[l + 1] - d[l]) / (2 * e[l]);
                long double r = hypotl(g, 1.0L);
                g = d[m] - d[l] + e[l] / (g + (g >= 0 ? fabsl(r) : -fabsl(r)));
                long double s = 1, c = 1, p = 0;
                int i;
                for (i = m - 1; i >= l; i--) {
                    long double f = s * e[i], b = c * e[i];
                    e[i + 1] = (r = hypotl(f, g));
                    if (r == 0) { d[i + 1] -= p; e[m] = 0; break; }
                    s = f / r; c = g / r;
                    g = d[i + 1] - p;
                    r = (d[i] - g) * s + 2 * c * b;
                    d[i + 1] = g + (p = s * r);
                    g = c * r - b;
                    f = z[i + 1];
                    z[i + 1] = s * z[i] + c * f;
                    z[i] = c * z[i] - s * f;
                }
                if (r == 0 && i >= l) continue;
                d[l] -= p; e[l] = g; e[m] = 0;
            }
        } while (m != l);
    }
}

static void sort_pairs(long double *u, long double *w, int n)
{
    for (int i = 1; i < n; i++)
        for (int j = i; j > 0 && u[j] < u[j - 1]; j--) {
            long double t = u[j]; u[j] = u[j - 1]; u[j - 1] = t;
            t = w[j]; w[j] = w[j - 1]; w[j - 1] = t;
        }
}

/* Rys nodes u (= t^2) and weights w, n <= 9. */
void oracle_rys_roots(int n, double x, double *u_out, double *w_out)
{
    long double d[NMAX], e[NMAX], z[NMAX];
    if (x > 40.0 + 5.0 * n) {
        /* half-range Hermite limit: 2n-point Gauss-Hermite, positive nodes */
        int N = 2 * n;
        long double hd[2 * NMAX], he[2 * NMAX], hz[2 * NMAX];
        for (int k = 0; k < N; k++) { hd[k] = 0; he[k] = k ? sqrtl(k / 2.0L) : 0; }
        tqli(hd, he, N, hz);
        long double s[NMAX], W[NMAX];
        int m = 0;
        for (int k = 0; k < N; k++)
            if (hd[k] > 0) { s[m] = hd[k]; W[m] = sqrtl(3.14159265358979323846264338327950288L) * hz[k] * hz[k]; m++; }
        sort_pairs(s, W, n);
        for (int i = 0; i < n; i++) {
            u_out[i] = (double)(s[i] * s[i] / x);
            w_out[i] = (double)(W[i] / sqrtl((long double)x));
        }
        return;
    }
    gl_init();
    /* discrete measure: nodes u_j = t_j^2, weights v_j exp(-x t_j^2) */
    static __thread long double un[NGL], vn[NGL], p0[NGL], p1[NGL];
    long double alpha[NMAX], beta[NMAX];
    for (int j = 0; j < NGL; j++) {
        un[j] = gl_t[j] * gl_t[j];
        vn[j] = gl_v[j] * expl(-(long double)x * un[j]);
        p0[j] = 0; p1[j] = 1;
    }
    long double nrm_prev = 1;
    for (int k = 0; k < n; k++) {
        long double nrm = 0, num = 0;
        for (int j = 0; j < NGL; j++) {
            long double pw = p1[j] * p1[j] * vn[j];
            nrm += pw; num += un[j] * pw;
        }
        alpha[k] = num / nrm;
        beta[k] = k ? nrm / nrm_prev : nrm;
        nrm_prev = nrm;
        for (int j = 0; j < NGL; j++) {
            long double pn = (un[j] - alpha[k]) * p1[j] - (k ? beta[k] : 0) * p0[j];
            p0[j] = p1[j]; p1[j] = pn;
        }
    }
    for (int k = 0; k < n; k++) { d[k] = alpha[k]; e[k] = k ? sqrtl(beta[k]) : 0; }
    tqli(d, e, n, z);
    long double wl[NMAX];
    for (int k = 0; k < n; k++) wl[k] = beta[0] * z[k] * z[k];
    sort_pairs(d, wl, n);
    for (int k = 0; k < n; k++) { u_out[k] = (double)d[k]; w_out[k] = (double)wl[k]; }
}

/* Boys function F_m(x), m = 0..mmax, by series + downward recursion (for tests). */
void oracle_boys(int mmax, double x, double *F)
{
    if (x > 300.0) {   /* exp(-x) below long-double resolution: F_m = (2m-1)/(2x) F_{m-1} */
        long double Fm = sqrtl(3.14159265358979323846264338327950288L / (4.0L * x));
        for (int m = 0; m <= mmax; m++) {
            F[m] = (double)Fm;
            Fm *= (2 * m + 1) / (2.0L * x);
        }
        return;
    }
    long double lx = x, ex = expl(-lx), term = 1.0L / (2 * mmax + 1), s = term;
    for (int k = 1; k < 200000; k++) {
        term *= 2 * lx / (2 * mmax + 2 * k + 1);
        s += term;
        if (term < s * 1e-21L) break;
    }
    long double Fm = s * ex;
    F[mmax] = (double)Fm;
    for (int m = mmax; m > 0; m--) {
        Fm = (2 * lx * Fm + ex) / (2 * m - 1);
        F[m - 1] = (double)Fm;
    }
}

static int ncart(int l) { return (l + 1) * (l + 2) / 2; }

static void cart_comp(int l, int n, int *lx, int *ly, int *lz)
{
    int c = 0;
    for (int a = l; a >= 0; a--)
        for (int b = l - a; b >= 0; b--) {
            if (c == n) { *lx = a; *ly = b; *lz = l - a - b; return; }
            c++;
        }
}

static double common_fac(int l)
{
    if (l == 0) return 0.282094791773878143;   /* 1/(2 sqrt(pi)) */
    if (l == 1) return 0.488602511902919921;   /* sqrt(3)/(2 sqrt(pi)) */
    return 1.0;
}

/* 2D integral table for one direction: I[i][j][k][l] with strides */
#define DIM 6   /* max index + 1 per centre: i up to LMAX+1 */

typedef struct {
    int li, lj, lk, ll, nci, ncj, nck, ncl, npi, npj, npk, npl;
    const double *ai, *aj, *ak, *al, *ci, *cj, *ck, *cl;
    const double *A, *B, *C, *D;
} quartet_t;

static void load_shell(const int *bas, const double *env, const int *atm, int sh,
                       int *l, int *np, int *nc, const double **a, const double **c, const double **R)
{
    const int *b = bas + sh * BAS_SLOTS;
    *l = b[ANG_OF]; *np = b[NPRIM_OF]; *nc = b[NCTR_OF];
    *a = env + b[PTR_EXP]; *c = env + b[PTR_COEFF];
    *R = env + atm[b[ATOM_OF] * ATM_SLOTS + PTR_COORD];
}

/*
 * Cartesian integrals of one shell quartet, all contractions.
 * deriv = 0: out[((((ci*ncj+cj)*nck+ck)*ncl+cl)*nfi+fi)... ] one component
 * deriv = 1: 3 components (x,y,z of d/dr1), component-major.
 * Layout: out[comp][ci][cj][ck][cl][fl][fk][fj][fi] flattened as
 *   comp*blk + ((((ci*ncj+cj)*nck+ck)*ncl+cl) * nf + ((fl*nfk+fk)*nfj+fj)*nfi+fi)
 */
static void shell_quartet(const quartet_t *q, int deriv, double *out)
{
    const int li = q->li, lj = q->lj, lk = q->lk, ll = q->ll;
    const int nfi = ncart(li), nfj = ncart(lj), nfk = ncart(lk), nfl = ncart(ll);
    const int nf = nfi * nfj * nfk * nfl;
    const int nctr = q->nci * q->ncj * q->nck * q->ncl;
    const int ncomp = deriv ? 3 : 1;
    const long blk = (long)nctr * nf;
    memset(out, 0, sizeof(double) * blk * ncomp);
    const int lij = li + lj + deriv, lkl = lk + ll;
    const int nroots = (li + lj + lk + ll + deriv) / 2 + 1;
    const double AB[3] = {q->A[0] - q->B[0], q->A[1] - q->B[1], q->A[2] - q->B[2]};
    const double CD[3] = {q->C[0] - q->D[0], q->C[1] - q->D[1], q->C[2] - q->D[2]};
    const double rab2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    const double rcd2 = CD[0] * CD[0] + CD[1] * CD[1] + CD[2] * CD[2];
    const double fac_sp = common_fac(li) * common_fac(lj) * common_fac(lk) * common_fac(ll);
    const double two_pi_52 = 34.986836655249725693;  /* 2 pi^(5/2) */

    /* G[dir][root][i][k] then HRR into H[dir][root][i][j][k][l] */
    static __thread double G[3][NMAX][DIM + LMAX + 1][2 * LMAX + 2];
    static __thread double H[3][NMAX][DIM][LMAX + 1][LMAX + 1][LMAX + 1];
    double *prim = (double *)malloc(sizeof(double) * nf * ncomp);

    for (int ip = 0; ip < q->npi; ip++)
    for (int jp = 0; jp < q->npj; jp++)
    for (int kp = 0; kp < q->npk; kp++)
    for (int lp = 0; lp < q->npl; lp++) {
        const double a = q->ai[ip], b = q->aj[jp], c = q->ak[kp], d = q->al[lp];
        const double p = a + b, qq = c + d;
        double P[3], Q[3], PQ[3];
        for (int x = 0; x < 3; x++) {
            P[x] = (a * q->A[x] + b * q->B[x]) / p;
            Q[x] = (c * q->C[x] + d * q->D[x]) / qq;
            PQ[x] = P[x] - Q[x];
        }
        const double rpq2 = PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2];
        const double rho = p * qq / (p + qq);
        const double T = rho * rpq2;
        const double pref = two_pi_52 / (p * qq * sqrt(p + qq))
                          * exp(-a * b / p * rab2) * exp(-c * d / qq * rcd2) * fac_sp;
        double u[NMAX], w[NMAX];
        oracle_rys_roots(nroots, T, u, w);
        for (int r = 0; r < nroots; r++) {
            const double B00 = 0.5 * u[r] / (p + qq);
            const double B10 = 0.5 / p * (1 - u[r] * qq / (p + qq));
            const double B01 = 0.5 / qq * (1 - u[r] * p / (p + qq));
            for (int x = 0; x < 3; x++) {
                const double C00 = (P[x] - q->A[x]) - u[r] * qq / (p + qq) * PQ[x];
                const double C01 = (Q[x] - q->C[x]) + u[r] * p / (p + qq) * PQ[x];
                double (*g)[2 * LMAX + 2] = G[x][r];
                g[0][0] = 1.0;
                for (int n = 0; n < lij; n++)
                    g[n + 1][0] = C00 * g[n][0] + (n ? n * B10 * g[n - 1][0] : 0.0);
                for (int m = 0; m < lkl; m++)
                    for (int n = 0; n <= lij; n++)
                        g[n][m + 1] = C01 * g[n][m] + (m ? m * B01 * g[n][m - 1] : 0.0)
                                    + (n ? n * B00 * g[n - 1][m] : 0.0);
                /* HRR on both sides: H[i][j][k][l] for i <= li+deriv */
                double t[DIM + LMAX + 1][LMAX + 1][2 * LMAX + 2];
                for (int n = 0; n <= lij; n++)
                    for (int m = 0; m <= lkl; m++) t[n][0][m] = g[n][m];
                for (int j = 1; j <= lj; j++)
                    for (int n = 0; n <= lij - j; n++)
                        for (int m = 0; m <= lkl; m++)
                            t[n][j][m] = t[n + 1][j - 1][m] + AB[x] * t[n][j - 1][m];
                for (int i = 0; i <= li + deriv; i++)
                    for (int j = 0; j <= lj; j++) {
                        double s[2 * LMAX + 2][LMAX + 1];
                        for (int m = 0; m <= lkl; m++) s[m][0] = t[i][j][m];
                        for (int l = 1; l <= ll; l++)
                            for (int m = 0; m <= lkl - l; m++)
                                s[m][l] = s[m + 1][l - 1] + CD[x] * s[m][l - 1];
                        for (int k = 0; k <= lk; k++)
                            for (int l = 0; l <= ll; l++) H[x][r][i][j][k][l] = s[k][l];
                    }
            }
        }
        /* primitive Cartesian block */
        for (int fl = 0; fl < nfl; fl++)
        for (int fk = 0; fk < nfk; fk++)
        for (int fj = 0; fj < nfj; fj++)
        for (int fi = 0; fi < nfi; fi++) {
            int ix, iy, iz, jx, jy, jz, kx, ky, kz, lx, ly, lz;
            cart_comp(li, fi, &ix, &iy, &iz); cart_comp(lj, fj, &jx, &jy, &jz);
            cart_comp(lk, fk, &kx, &ky, &kz); cart_comp(ll, fl, &lx, &ly, &lz);
            const int f = ((fl * nfk + fk) * nfj + fj) * nfi + fi;
            if (!deriv) {
                double acc = 0;
                for (int r = 0; r < nroots; r++)
                    acc += w[r] * H[0][r][ix][jx][kx][lx] * H[1][r][iy][jy][ky][ly] * H[2][r][iz][jz][kz][lz];
                prim[f] = acc * pref;
            } else {
                double sx = 0, sy = 0, sz = 0;
                for (int r = 0; r < nroots; r++) {
                    double hx = H[0][r][ix][jx][kx][lx], hy = H[1][r][iy][jy][ky][ly], hz = H[2][r][iz][jz][kz][lz];
                    double dx = -2 * a * H[0][r][ix + 1][jx][kx][lx] + (ix ? ix * H[0][r][ix - 1][jx][kx][lx] : 0);
                    double dy = -2 * a * H[1][r][iy + 1][jy][ky][ly] + (iy ? iy * H[1][r][iy - 1][jy][ky][ly] : 0);
                    double dz = -2 * a * H[2][r][iz + 1][jz][kz][lz] + (iz ? iz * H[2][r][iz - 1][jz][kz][lz] : 0);
                    sx += w[r] * dx * hy * hz;
                    sy += w[r] * hx * dy * hz;
                    sz += w[r] * hx * hy * dz;
                }
                prim[f] = sx * pref; prim[nf + f] = sy * pref; prim[2 * nf + f] = sz * pref;
            }
        }
        /* contract into every contraction combination */
        for (int ci = 0; ci < q->nci; ci++)
        for (int cj = 0; cj < q->ncj; cj++)
        for (int ck = 0; ck < q->nck; ck++)
        for (int cl = 0; cl < q->ncl; cl++) {
            const double cc = q->ci[ci * q->npi + ip] * q->cj[cj * q->npj + jp]
                            * q->ck[ck * q->npk + kp] * q->cl[cl * q->npl + lp];
            const long base = ((((long)ci * q->ncj + cj) * q->nck + ck) * q->ncl + cl) * nf;
            for (int comp = 0; comp < ncomp; comp++)
                for (int f = 0; f < nf; f++)
                    out[comp * blk + base + f] += cc * prim[comp * nf + f];
        }
    }
    free(prim);
}

/*
 * Cartesian s2kl block, the oracle counterpart of compute_int2e_gpu /
 * compute_int2e_ip1_gpu on a Cartesian molecule:
 *   out[comp][fi_local][j][k*(k+1)/2 + l],  k >= l,
 * i over shells [b0, b1), j, k, l over all shells; AO offsets from ao_loc
 * (Cartesian, nctr-aware).  Parallel over i-shell x j-shell pairs.
 */
int oracle_eri_s2kl(const int *atm, int natm, const int *bas, int nbas, const double *env,
                    const int *ao_loc, int b0, int b1, int deriv, double *out)
{
    (void)natm;
    const int nao = ao_loc[nbas];
    const long nao_pair = (long)nao * (nao + 1) / 2;
    const int nfblk = ao_loc[b1] - ao_loc[b0];
    const int ncomp = deriv ? 3 : 1;
    const long comp_stride = (long)nfblk * nao * nao_pair;
    memset(out, 0, sizeof(double) * comp_stride * ncomp);
    const int npairs = (b1 - b0) * nbas;
#pragma omp parallel for schedule(dynamic)
    for (int ij = 0; ij < npairs; ij++) {
        const int ish = b0 + ij / nbas, jsh = ij % nbas;
        for (int ksh = 0; ksh < nbas; ksh++)
            for (int lsh = 0; lsh <= ksh; lsh++) {
                quartet_t q;
                load_shell(bas, env, atm, ish, &q.li, &q.npi, &q.nci, &q.ai, &q.ci, &q.A);
                load_shell(bas, env, atm, jsh, &q.lj, &q.npj, &q.ncj, &q.aj, &q.cj, &q.B);
                load_shell(bas, env, atm, ksh, &q.lk, &q.npk, &q.nck, &q.ak, &q.ck, &q.C);
                load_shell(bas, env, atm, lsh, &q.ll, &q.npl, &q.ncl, &q.al, &q.cl, &q.D);
                const int nfi = ncart(q.li), nfj = ncart(q.lj), nfk = ncart(q.lk), nfl = ncart(q.ll);
                const int nf = nfi * nfj * nfk * nfl;
                const long blk = (long)q.nci * q.ncj * q.nck * q.ncl * nf;
                double *qb = (double *)malloc(sizeof(double) * blk * ncomp);
                shell_quartet(&q, deriv, qb);
                for (int ci = 0; ci < q.nci; ci++)
                for (int cj = 0; cj < q.ncj; cj++)
                for (int ck = 0; ck < q.nck; ck++)
                for (int cl = 0; cl < q.ncl; cl++) {
                    const long base = ((((long)ci * q.ncj + cj) * q.nck + ck) * q.ncl + cl) * nf;
                    for (int fl = 0; fl < nfl; fl++)
                    for (int fk = 0; fk < nfk; fk++) {
                        const int k = ao_loc[ksh] + ck * nfk + fk, l = ao_loc[lsh] + cl * nfl + fl;
                        if (l > k) continue;
                        const long kl = (long)k * (k + 1) / 2 + l;
                        for (int fj = 0; fj < nfj; fj++)
                        for (int fi = 0; fi < nfi; fi++) {
                            const int i = ao_loc[ish] + ci * nfi + fi - ao_loc[b0];
                            const int j = ao_loc[jsh] + cj * nfj + fj;
                            const int f = ((fl * nfk + fk) * nfj + fj) * nfi + fi;
                            for (int comp = 0; comp < ncomp; comp++)
                                out[comp * comp_stride + ((long)i * nao + j) * nao_pair + kl] = qb[comp * blk + base + f];
                        }
                    }
                }
                free(qb);
            }
    }
    return 0;
}

/* One shell quartet, all contractions, layout of shell_quartet (for tests). */
int oracle_eri_quartet(const int *atm, const int *bas, const double *env,
                       int ish, int jsh, int ksh, int lsh, int deriv, double *out)
{
    quartet_t q;
    load_shell(bas, env, atm, ish, &q.li, &q.npi, &q.nci, &q.ai, &q.ci, &q.A);
    load_shell(bas, env, atm, jsh, &q.lj, &q.npj, &q.ncj, &q.aj, &q.cj, &q.B);
    load_shell(bas, env, atm, ksh, &q.lk, &q.npk, &q.nck, &q.ak, &q.ck, &q.C);
    load_shell(bas, env, atm, lsh, &q.ll, &q.npl, &q.ncl, &q.al, &q.cl, &q.D);
    shell_quartet(&q, deriv, out);
    return 0;
}

int oracle_eri_quartet(const int *atm, const int *bas, const double *env,
                       int ish, int jsh, int ksh, int lsh, int deriv, double *out);

/* Two checksums per quartet and component, same definition as
 * ccsd_b200_eri_quartet_checksums; decontracted shells only. */
int oracle_eri_quartet_checksums(int deriv, const int *atm, const int *bas, const double *env,
                                 const int *quartets, long nq, double *qsum)
{
    const int ncomp = deriv ? 3 : 1;
    gl_init();
#pragma omp parallel for schedule(dynamic, 16)
    for (long q = 0; q < nq; q++) {
        const int *s = quartets + 4 * q;
        int nf = 1;
        for (int t = 0; t < 4; t++) nf *= ncart(bas[s[t] * BAS_SLOTS + ANG_OF]);
        double *buf = (double *)malloc(sizeof(double) * nf * ncomp);
        oracle_eri_quartet(atm, bas, env, s[0], s[1], s[2], s[3], deriv, buf);
        const int nfi = ncart(bas[s[0] * BAS_SLOTS + ANG_OF]), nfj = ncart(bas[s[1] * BAS_SLOTS + ANG_OF]);
        const int nfk = ncart(bas[s[2] * BAS_SLOTS + ANG_OF]), nfl = ncart(bas[s[3] * BAS_SLOTS + ANG_OF]);
        for (int c = 0; c < ncomp; c++) {
            double s1 = 0, s2 = 0;
            int f = 0;
            for (int fi = 0; fi < nfi; fi++)
                for (int fj = 0; fj < nfj; fj++)
                    for (int fk = 0; fk < nfk; fk++)
                        for (int fl = 0; fl < nfl; fl++, f++) {
                            const double v = buf[c * nf + ((fl * nfk + fk) * nfj + fj) * nfi + fi];
                            s1 += v * (1.0 + 0.125 * (f & 7));
                            s2 += v * v;
                        }
            qsum[(q * ncomp + c) * 2] = s1;
            qsum[(q * ncomp + c) * 2 + 1] = s2;
        }
        free(buf);
    }
    return 0;
}
