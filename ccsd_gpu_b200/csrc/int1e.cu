// One-electron integrals and their first derivatives over Cartesian shells, sm_100a.
//
// Replaces the libcint calls of the gradient's one-electron terms and of the
// SCF set-up: mol.intor("int1e_ovlp" / "int1e_kin" / "int1e_nuc") and the
// derivative forms "int1e_ipovlp", "int1e_ipkin", "int1e_ipnuc",
// "int1e_iprinv" used by hcore_generator / get_ovlp
// (ref: ccsd_gpu/gpu_ccsd_grad.py:554-584).
//
// One thread per (i, j) shell pair of the decontracted basis.  Per primitive pair:
//   * overlap and kinetic from the 1D Obara-Saika tables
//       S(a+1,b) = PA S(a,b) + (a S(a-1,b) + b S(a,b-1)) / 2p,  S(a,b+1) likewise with PB,
//       K(a,b)   = -1/2 [ b(b-1) S(a,b-2) - 2 beta (2b+1) S(a,b) + 4 beta^2 S(a,b+2) ];
//   * 1/|r - C| by Rys quadrature: per root u, the 1D table
//       I(a+1,0) = C00 I(a,0) + a B10 I(a-1,0),  C00 = PA - u PC,  B10 = (1 - u)/2p,
//       I(a,b+1) = I(a+1,b) + (A - B) I(a,b),
//     prefactor 2 pi / p exp(-alpha beta/p |AB|^2), Rys argument p |PC|^2.
// Bra derivative ("ip", d/dr on the first function): D I(a) = a I(a-1) - 2 alpha I(a+1).
// Output: full Cartesian (ncomp, nao, nao) matrix; libcint normalisation
// (coefficients from env, angular factor for s and p).
#include "common.cuh"
#include "rys.cuh"

namespace cb {

enum { OP_OVLP = 0, OP_KIN = 1, OP_NUC = 2, OP_RINV = 3, OP_IPOVLP = 4, OP_IPKIN = 5, OP_IPNUC = 6, OP_IPRINV = 7 };

static constexpr int L1 = CB_LMAX + 1;      // bra index range incl. derivative
static constexpr int NA = CB_LMAX + 2;      // a <= l_i + 1
static constexpr int NB = CB_LMAX + 3;      // b <= l_j + 2

__device__ __forceinline__ double cfac(int l)
{
    return l == 0 ? 0.282094791773878143 : (l == 1 ? 0.488602511902919921 : 1.0);
}

__device__ __forceinline__ void cart_xyz(int l, int n, int &x, int &y, int &z)
{
    int c = 0;
    for (int a = l; a >= 0; a--)
        for (int b = l - a; b >= 0; b--) {
            if (c == n) { x = a; y = b; z = l - a - b; return; }
            c++;
        }
    x = y = z = 0;
}

__global__ void int1e_kernel(int op, const int *__restrict__ atm, int natm, const int *__restrict__ bas, int nbas,
                             const double *__restrict__ env, const int *__restrict__ ao_loc, int origin_atom,
                             double *__restrict__ out)
{
    const long long pair = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (pair >= (long long)nbas * nbas) return;
    const int ish = (int)(pair / nbas), jsh = (int)(pair % nbas);
    const int *bi = bas + ish * CB_BAS_SLOTS, *bj = bas + jsh * CB_BAS_SLOTS;
    const int li = bi[CB_ANG_OF], lj = bj[CB_ANG_OF], npi = bi[CB_NPRIM_OF], npj = bj[CB_NPRIM_OF];
    const double *ai_ = env + bi[CB_PTR_EXP], *aj_ = env + bj[CB_PTR_EXP];
    const double *ci_ = env + bi[CB_PTR_COEFF], *cj_ = env + bj[CB_PTR_COEFF];
    const double *A = env + atm[bi[CB_ATOM_OF] * CB_ATM_SLOTS + CB_PTR_COORD];
    const double *B = env + atm[bj[CB_ATOM_OF] * CB_ATM_SLOTS + CB_PTR_COORD];
    const bool deriv = op >= OP_IPOVLP;
    const int base = deriv ? op - OP_IPOVLP : op;
    const int ncomp = deriv ? 3 : 1;
    const int nfi = ncart(li), nfj = ncart(lj);
    const int nao = ao_loc[nbas];
    const int i0 = ao_loc[ish], j0 = ao_loc[jsh];
    double acc[3][15][15];
    for (int c = 0; c < ncomp; c++)
        for (int fi = 0; fi < nfi; fi++)
            for (int fj = 0; fj < nfj; fj++) acc[c][fi][fj] = 0.0;
    const double AB[3] = {A[0] - B[0], A[1] - B[1], A[2] - B[2]};
    const double rab2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    const double fac = cfac(li) * cfac(lj);
    const int amax = li + (deriv ? 1 : 0);

    for (int ip = 0; ip < npi; ip++)
        for (int jp = 0; jp < npj; jp++) {
            const double a = ai_[ip], b = aj_[jp], p = a + b;
            const double cc = ci_[ip] * cj_[jp] * fac;
            const double kab = exp(-a * b / p * rab2);
            double P[3];
            for (int x = 0; x < 3; x++) P[x] = (a * A[x] + b * B[x]) / p;
            if (base == OP_OVLP || base == OP_KIN) {
                // 1D overlap tables S[dir][a][b], b up to lj + 2 (kinetic)
                double S[3][NA][NB];
                const int bmax = lj + (base == OP_KIN ? 2 : 0);
                for (int x = 0; x < 3; x++) {
                    const double PA = P[x] - A[x], PB = P[x] - B[x], h = 0.5 / p;
                    S[x][0][0] = sqrt(M_PI / p) * (x == 0 ? kab : 1.0);
                    for (int i = 0; i < amax; i++)
                        S[x][i + 1][0] = PA * S[x][i][0] + (i ? i * h * S[x][i - 1][0] : 0.0);
                    for (int j = 0; j < bmax; j++)
                        for (int i = 0; i <= amax; i++)
                            S[x][i][j + 1] = PB * S[x][i][j] + h * ((i ? i * S[x][i - 1][j] : 0.0) +
                                                                    (j ? j * S[x][i][j - 1] : 0.0));
                }
                for (int fi = 0; fi < nfi; fi++) {
                    int e[3];
                    cart_xyz(li, fi, e[0], e[1], e[2]);
                    for (int fj = 0; fj < nfj; fj++) {
                        int f[3];
                        cart_xyz(lj, fj, f[0], f[1], f[2]);
                        double s[3], k[3], ds[3], dk[3];
                        for (int x = 0; x < 3; x++) {
                            const int ia = e[x], jb = f[x];
                            s[x] = S[x][ia][jb];
                            if (base == OP_KIN)
                                k[x] = -0.5 * ((jb > 1 ? jb * (jb - 1) * S[x][ia][jb - 2] : 0.0) -
                                               2 * b * (2 * jb + 1) * S[x][ia][jb] + 4 * b * b * S[x][ia][jb + 2]);
                            if (deriv) {
                                ds[x] = -2 * a * S[x][ia + 1][jb] + (ia ? ia * S[x][ia - 1][jb] : 0.0);
                                if (base == OP_KIN) {
                                    auto kk = [&](int aa) {
                                        return -0.5 * ((jb > 1 ? jb * (jb - 1) * S[x][aa][jb - 2] : 0.0) -
                                                       2 * b * (2 * jb + 1) * S[x][aa][jb] +
                                                       4 * b * b * S[x][aa][jb + 2]);
                                    };
                                    dk[x] = -2 * a * kk(ia + 1) + (ia ? ia * kk(ia - 1) : 0.0);
                                }
                            }
                        }
                        for (int c = 0; c < ncomp; c++) {
                            double v;
                            if (!deriv) {
                                v = base == OP_OVLP ? s[0] * s[1] * s[2]
                                                    : k[0] * s[1] * s[2] + s[0] * k[1] * s[2] + s[0] * s[1] * k[2];
                            } else {
                                double t[3] = {s[0], s[1], s[2]};
                                t[c] = ds[c];
                                if (base == OP_OVLP) {
                                    v = t[0] * t[1] * t[2];
                                } else {
                                    // d/dr_c of T: the derivative acts on the bra factor of direction c
                                    double kt[3] = {k[0], k[1], k[2]};
                                    kt[c] = dk[c];
                                    v = kt[0] * t[1] * t[2] + t[0] * kt[1] * t[2] + t[0] * t[1] * kt[2];
                                }
                            }
                            acc[c][fi][fj] += cc * v;
                        }
                    }
                }
            } else {
                // nuclear attraction (sum over nuclei, -Z) or 1/|r - C| at one atom
                const int c0 = base == OP_NUC ? 0 : origin_atom;
                const int c1 = base == OP_NUC ? natm : origin_atom + 1;
                const int nroots = (li + lj + (deriv ? 1 : 0)) / 2 + 1;
                for (int ic = c0; ic < c1; ic++) {
                    const double *C = env + atm[ic * CB_ATM_SLOTS + CB_PTR_COORD];
                    const double z = base == OP_NUC ? -(double)atm[ic * CB_ATM_SLOTS] : 1.0;
                    double PC[3];
                    for (int x = 0; x < 3; x++) PC[x] = P[x] - C[x];
                    const double T = p * (PC[0] * PC[0] + PC[1] * PC[1] + PC[2] * PC[2]);
                    double u[RYS_NROOTS_MAX], w[RYS_NROOTS_MAX];
                    rys_roots(nroots, T, u, w);
                    const double pref = 2.0 * M_PI / p * kab * z;
                    for (int r = 0; r < nroots; r++) {
                        double I[3][NA + CB_LMAX][L1];
                        const int lij = amax + lj;
                        for (int x = 0; x < 3; x++) {
                            const double c00 = (P[x] - A[x]) - u[r] * PC[x];
                            const double b10 = (1.0 - u[r]) * 0.5 / p;
                            double v[NA + CB_LMAX];
                            v[0] = x == 0 ? w[r] * pref : 1.0;
                            for (int n = 0; n < lij; n++) v[n + 1] = c00 * v[n] + (n ? n * b10 * v[n - 1] : 0.0);
                            for (int n = 0; n <= lij; n++) I[x][n][0] = v[n];
                            for (int j = 1; j <= lj; j++)
                                for (int n = 0; n <= lij - j; n++)
                                    I[x][n][j] = I[x][n + 1][j - 1] + AB[x] * I[x][n][j - 1];
                        }
                        for (int fi = 0; fi < nfi; fi++) {
                            int e[3];
                            cart_xyz(li, fi, e[0], e[1], e[2]);
                            for (int fj = 0; fj < nfj; fj++) {
                                int f[3];
                                cart_xyz(lj, fj, f[0], f[1], f[2]);
                                for (int c = 0; c < ncomp; c++) {
                                    double t[3];
                                    for (int x = 0; x < 3; x++) {
                                        const int ia = e[x], jb = f[x];
                                        if (deriv && x == c)
                                            t[x] = -2 * a * I[x][ia + 1][jb] + (ia ? ia * I[x][ia - 1][jb] : 0.0);
                                        else
                                            t[x] = I[x][ia][jb];
                                    }
                                    acc[c][fi][fj] += cc * t[0] * t[1] * t[2];
                                }
                            }
                        }
                    }
                }
            }
        }
    for (int c = 0; c < ncomp; c++)
        for (int fi = 0; fi < nfi; fi++)
            for (int fj = 0; fj < nfj; fj++)
                out[((long long)c * nao + i0 + fi) * nao + j0 + fj] = acc[c][fi][fj];
}

}  // namespace cb

extern "C" int ccsd_b200_int1e_cart(int op, const int32_t *atm, int natm, const int32_t *bas, int nbas,
                                    const double *env, const int32_t *ao_loc, int lmax, int origin_atom,
                                    double *out, void *stream)
{
    if (op < 0 || op > 7 || !atm || natm <= 0 || !bas || nbas <= 0 || !env || !ao_loc || !out || lmax < 0 ||
        ((op == 3 || op == 7) && (origin_atom < 0 || origin_atom >= natm))) {
        cb::set_error("ccsd_b200_int1e_cart: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    if (lmax > CB_LMAX) {
        cb::set_error("ccsd_b200_int1e_cart: l = %d > %d is not supported", lmax, CB_LMAX);
        return CCSD_B200_ERR_UNSUPPORTED;
    }
    const long long npair = (long long)nbas * nbas;
    const int bs = 64;
    cb::int1e_kernel<<<(int)((npair + bs - 1) / bs), bs, 0, (cudaStream_t)stream>>>(op, atm, natm, bas, nbas, env,
                                                                                   ao_loc, origin_atom, out);
    return cb::check_launch("int1e_kernel");
}
