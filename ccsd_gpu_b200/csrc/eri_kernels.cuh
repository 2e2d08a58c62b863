// Rys-quadrature two-electron integrals and their first derivatives, sm_100a.
//
// Replaces fill_int2e_kernel / fill_int2e_ip1_kernel and their launch loops
// (ref: ccsd_gpu/cuda/int2e_module.py:130-463, ccsd_gpu/cuda/int2e_ip1_module.py:273-667,
//  ccsd_gpu/cuda/int2e_gpu.py:39-108, ccsd_gpu/cuda/int2e_ip1_gpu.py:148-216).
//
// Work decomposition (one warp = one shell quartet, no block-wide barriers):
//   slot   = (primitive quartet, Rys root); a warp processes its quartet's slots in
//            batches that fit its shared-memory slice;
//   phase A  lanes over primitive quartets: Gaussian-product data and the Rys
//            nodes/weights (each lane evaluates its own roots from the tables);
//   phase B  lanes over (slot, direction): 2D recurrences + both horizontal
//            transfers for one Cartesian direction, written to shared memory;
//   phase C  lanes over output functions: accumulate gx*gy*gz (or the
//            derivative combination) in registers across all slots.
// The warp's outputs stay in registers until the quartet is finished, so the
// output is written once.  Output functions are enumerated with the l-index
// fastest so neighbouring lanes write neighbouring kl-pair addresses.
//
// This header holds the device code and the kernel templates; each
// eri_inst_*.cu translation unit instantiates the launchers of one
// (derivative order, angular-momentum range) so the variants compile in
// parallel, and eri.cu holds the C entry points.
#pragma once
#include "common.cuh"
#include "eri_launch.h"
#include "rys.cuh"

namespace cb {


// Cartesian exponents, lexicographic order per l (l <= 4), packed x | y<<4 | z<<8
__constant__ uint16_t c_cart[35] = {
    0x000,
    0x001, 0x010, 0x100,
    0x002, 0x011, 0x101, 0x020, 0x110, 0x200,
    0x003, 0x012, 0x102, 0x021, 0x111, 0x201, 0x030, 0x120, 0x210, 0x300,
    0x004, 0x013, 0x103, 0x022, 0x112, 0x202, 0x031, 0x121, 0x211, 0x301,
    0x040, 0x130, 0x220, 0x310, 0x400};
__constant__ int c_cart_off[5] = {0, 1, 4, 10, 20};

struct Shell {
    int l, np;
    const double *exps, *coefs;
    double R[3];
};

__device__ __forceinline__ Shell load_shell(const int *__restrict__ atm, const int *__restrict__ bas,
                                            const double *__restrict__ env, int sh)
{
    Shell s;
    const int *b = bas + sh * CB_BAS_SLOTS;
    s.l = b[CB_ANG_OF];
    s.np = b[CB_NPRIM_OF];
    s.exps = env + b[CB_PTR_EXP];
    s.coefs = env + b[CB_PTR_COEFF];
    const double *r = env + atm[b[CB_ATOM_OF] * CB_ATM_SLOTS + CB_PTR_COORD];
    s.R[0] = r[0];
    s.R[1] = r[1];
    s.R[2] = r[2];
    return s;
}

// Primitive-pair screen.  A pair of Gaussians with exponents a, b on centres
// A, B carries exp(-ab/(a+b) |AB|^2) in every integral it enters; the pair is
// dropped when ab/(a+b) |AB|^2 > kPairCut + (la + lb) ln(1 + |AB|), the second
// term allowing for the polynomial factors (P-A)^i (P-B)^j of the pair's
// Cartesian functions (|P-A|, |P-B| <= |AB|).  e^-50 ~ 2e-22 relative to an
// O(1) normalised primitive product: far below FP64 resolution of any block.
// The kept pairs of one shell pair are a 128-bit mask in registers (bit
// ia * nb + ib), built with warp ballots; pairs beyond 128 are not screened.
static constexpr double kPairCut = 50.0;

struct PairMask {
    unsigned w[4];
    int n;      // kept pairs
    int nb;     // primitives of the second shell
    int all;    // more than 128 pairs: every pair kept, index decoded directly
};

// Every lane of the calling warp must be active (warp ballots).
__device__ __forceinline__ PairMask pair_mask(const Shell &a, const Shell &b, double r2, int lsum)
{
    PairMask m;
    const int n = a.np * b.np;
    m.nb = b.np;
    m.all = n > 128;
    m.n = m.all ? n : 0;
    const double cut = kPairCut + lsum * log1p(sqrt(r2));
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int c = 0; c < 4; c++) {
        const int t = c * 32 + lane;
        bool keep = false;
        if (!m.all && t < n) {
            const int ia = t / b.np, ib = t - ia * b.np;
            const double ea = a.exps[ia], eb = b.exps[ib];
            keep = ea * eb / (ea + eb) * r2 <= cut;
        }
        m.w[c] = __ballot_sync(0xffffffffu, keep);
        if (!m.all) m.n += __popc(m.w[c]);
    }
    return m;
}

// Position of the k-th (0-based) set bit of w; w has more than k set bits.
__device__ __forceinline__ int nth_set_bit(unsigned w, int k)
{
    int pos = 0;
#pragma unroll
    for (int half = 16; half > 0; half >>= 1) {
        const unsigned lo = w & ((1u << half) - 1u);
        const int c = __popc(lo);
        if (k >= c) {
            k -= c;
            w >>= half;
            pos += half;
        } else {
            w = lo;
        }
    }
    return pos;
}

// Primitive indices of the k-th kept pair.
__device__ __forceinline__ void kept_pair(const PairMask &m, int k, int &ia, int &ib)
{
    int t = k;
    if (!m.all) {
        int c = 0;
        while (c < 3) {
            const int pc = __popc(m.w[c]);
            if (k < pc) break;
            k -= pc;
            c++;
        }
        t = c * 32 + nth_set_bit(m.w[c], k);
    }
    ia = t / m.nb;
    ib = t - ia * m.nb;
}


// ---- Gaussian-product data of the kept primitive pairs (phase A, part 1) ----
// One row of kPairStride doubles per kept primitive pair of a shell pair
// (a, b), with R = A - B and r2 = |R|^2:
//   [0..2] P - A = -b/(a+b) R,  [3] a+b,  [4] 1/(2(a+b)),
//   [5] c_a c_b exp(-ab/(a+b) r2) / (a+b),  [6] 2a (the ip1 factor of the bra).
// A quartet builds the rows of its bra and ket pairs once (lanes over pairs),
// so the per-slot work below has one division and one square root instead of
// the ~8 divisions and the exponential of the direct evaluation.
static constexpr int kPairStride = 8;
// The pair rows of a quartet are kept in shared memory when, beside them, a
// batch of at least min(nslot, 32) slots still fits (per_slot doubles each);
// otherwise each slot computes its two rows on the fly (two exponentials and
// divisions per slot).  Long general contractions (9 x 9 primitive pairs of
// an oxygen s shell in cc-pVDZ: 1296 doubles) keep their table this way.
__device__ __forceinline__ bool pair_table_fits(int tabn, int room, int per_slot, int nslot)
{
    const int batch = nslot < 32 ? (nslot > 1 ? nslot : 1) : 32;
    return tabn <= room - batch * per_slot;
}

__device__ __forceinline__ void pair_row(const Shell &a, const Shell &b, const PairMask &m, int k,
                                         const double *__restrict__ R, double r2, double *__restrict__ p)
{
    int ia, ib;
    kept_pair(m, k, ia, ib);
    const double ea = a.exps[ia], eb = b.exps[ib];
    const double sab = ea + eb, is = 1.0 / sab;
    p[0] = -eb * is * R[0];
    p[1] = -eb * is * R[1];
    p[2] = -eb * is * R[2];
    p[3] = sab;
    p[4] = 0.5 * is;
    p[5] = a.coefs[ia] * b.coefs[ib] * exp(-ea * eb * is * r2) * is;
    p[6] = 2.0 * ea;
    p[7] = 0.0;
}

// Pair rows of both pairs into tab (bra rows first, then ket rows);
// threads tid, tid + nt, ... of the cooperating group.
__device__ __forceinline__ void build_pair_tables(const Shell &si, const Shell &sj, const Shell &sk,
                                                  const Shell &sl, const PairMask &mb, const PairMask &mk,
                                                  const double *__restrict__ AB, double rab2,
                                                  const double *__restrict__ CD, double rcd2,
                                                  double *__restrict__ tab, int tid, int nt)
{
    for (int k = tid; k < mb.n + mk.n; k += nt) {
        if (k < mb.n)
            pair_row(si, sj, mb, k, AB, rab2, tab + k * kPairStride);
        else
            pair_row(sk, sl, mk, k - mb.n, CD, rcd2, tab + k * kPairStride);
    }
}

// ---- slot parameters (phase A, part 2) ----
// Slots s in [s0, s1) (slot = primitive quartet pq * nroots + root r), one
// per thread: Rys node/weight r of pq and the recurrence coefficients,
// written to par[(s - s0) * kParStride + 0..10].  With tab == nullptr the
// pair rows are computed here (contractions too long for the table).
__device__ __forceinline__ void slot_params(const double *__restrict__ tab, const Shell &si, const Shell &sj,
                                            const Shell &sk, const Shell &sl, const PairMask &mb,
                                            const PairMask &mk, const double *__restrict__ AB, double rab2,
                                            const double *__restrict__ CD, double rcd2, int nroots, double pref0,
                                            int s0, int s1, double *__restrict__ par, int tid, int nt)
{
    for (int s = s0 + tid; s < s1; s += nt) {
        const int pq = s / nroots, r = s - pq * nroots;
        const int ib = pq / mk.n, ik = pq - ib * mk.n;
        double bl[kPairStride], kl[kPairStride];
        const double *bp, *kp;
        if (tab) {
            bp = tab + ib * kPairStride;
            kp = tab + (mb.n + ik) * kPairStride;
        } else {
            pair_row(si, sj, mb, ib, AB, rab2, bl);
            pair_row(sk, sl, mk, ik, CD, rcd2, kl);
            bp = bl;
            kp = kl;
        }
        const double aij = bp[3], akl = kp[3];
        const double inv = 1.0 / (aij + akl);
        double PQ[3];
#pragma unroll
        for (int x = 0; x < 3; x++) PQ[x] = (si.R[x] + bp[x]) - (sk.R[x] + kp[x]);
        const double rpq2 = PQ[0] * PQ[0] + PQ[1] * PQ[1] + PQ[2] * PQ[2];
        double u, w;
        rys_node(nroots, r, aij * akl * inv * rpq2, u, w);
        double *p = par + (s - s0) * kParStride;
        const double ua = u * inv;
#pragma unroll
        for (int x = 0; x < 3; x++) {
            p[x] = bp[x] - ua * akl * PQ[x];
            p[3 + x] = kp[x] + ua * aij * PQ[x];
        }
        p[6] = 0.5 * ua;
        p[7] = bp[4] * (1.0 - ua * akl);
        p[8] = kp[4] * (1.0 - ua * aij);
        p[9] = w * pref0 * bp[5] * kp[5] * sqrt(inv);
        p[10] = bp[6];
    }
}

__device__ __forceinline__ double common_fac(int l)
{
    return l == 0 ? 0.282094791773878143 : (l == 1 ? 0.488602511902919921 : 1.0);
}

// One Cartesian direction of one slot: 2D recurrences then HRR on both pairs.
// Result g[i + j*sj + k*sk + l*sl], i <= li+D, j <= lj, k <= lk, l <= ll.
template <int D>
__device__ void build_g(const double *__restrict__ p, int dir, int li, int lj, int lk, int ll,
                        double ab, double cd, double *__restrict__ g)
{
    const int lij = li + lj + D, lkl = lk + ll;
    const int sj = li + 1 + D, sk = sj * (lj + 1), sl = sk * (lk + 1);
    const double c00 = p[dir], c01 = p[3 + dir], b00 = p[6], b10 = p[7], b01 = p[8];
    double t[2 * CB_LMAX + 2][2 * CB_LMAX + 1];   // t[n][m], n <= lij, m <= lkl
    t[0][0] = dir == 0 ? p[9] : 1.0;
    if (lij > 0) t[1][0] = c00 * t[0][0];
    for (int n = 1; n < lij; n++) t[n + 1][0] = c00 * t[n][0] + n * b10 * t[n - 1][0];
    for (int m = 0; m < lkl; m++) {
        const double mb = m * b01;
        t[0][m + 1] = c01 * t[0][m] + (m ? mb * t[0][m - 1] : 0.0);
        for (int n = 1; n <= lij; n++)
            t[n][m + 1] = c01 * t[n][m] + (m ? mb * t[n][m - 1] : 0.0) + n * b00 * t[n - 1][m];
    }
    // HRR on (i,j): in place, column m at a time; values for j land in g at
    // i + j*sj + m*sk (fits because sk*(lkl+1) <= sk*(lk+1)*(ll+1)).
    for (int m = 0; m <= lkl; m++) {
        double v[2 * CB_LMAX + 2];
        for (int n = 0; n <= lij; n++) v[n] = t[n][m];
        for (int i = 0; i <= li + D; i++) g[i + m * sk] = v[i];
        for (int j = 1; j <= lj; j++) {
            for (int n = 0; n <= lij - j; n++) v[n] = v[n + 1] + ab * v[n];
            for (int i = 0; i <= li + D; i++) g[i + j * sj + m * sk] = v[i];
        }
    }
    // HRR on (k,l): per (i,j) column, all writes stay inside the same column
    if (ll > 0) {
        for (int o = 0; o < sk; o++) {
            double w[2 * CB_LMAX + 1];
            for (int m = 0; m <= lkl; m++) w[m] = g[o + m * sk];
            for (int l = 1; l <= ll; l++) {
                for (int m = 0; m <= lkl - l; m++) w[m] = w[m + 1] + cd * w[m];
                for (int k = 0; k <= lk; k++) g[o + k * sk + l * sl] = w[k];
            }
        }
    }
}

// Same recurrences as build_g with compile-time angular momenta (l <= 2),
// streamed: the transfer recurrence keeps two columns (m-1, m) of the 2D table
// in registers, each finished column goes through the (i,j) horizontal
// recurrence straight into shared memory, and the (k,l) horizontal recurrence
// runs per (i,j) column from there.  Peak live state is ~4 (LIJ+1) doubles.
template <int D, int LI, int LJ, int LK, int LL>
__device__ __noinline__ void build_g_fixed(const double *__restrict__ p, int dir, double ab, double cd,
                                              double *__restrict__ g)
{
    constexpr int LIJ = LI + LJ + D, LKL = LK + LL;
    constexpr int SJ = LI + 1 + D, SK = SJ * (LJ + 1), SL = SK * (LK + 1);
    const double c00 = p[dir], c01 = p[3 + dir], b00 = p[6], b10 = p[7], b01 = p[8];
    double prev[LIJ + 1], cur[LIJ + 1];
    cur[0] = dir == 0 ? p[9] : 1.0;
#pragma unroll
    for (int n = 0; n < LIJ; n++) cur[n + 1] = c00 * cur[n] + (n ? n * b10 * cur[n - 1] : 0.0);
#pragma unroll
    for (int n = 0; n <= LIJ; n++) prev[n] = 0.0;
#pragma unroll
    for (int m = 0; m <= LKL; m++) {
        {   // HRR (i,j) of column m into g[i + j*SJ + m*SK]
            double v[LIJ + 1];
#pragma unroll
            for (int n = 0; n <= LIJ; n++) v[n] = cur[n];
#pragma unroll
            for (int i = 0; i <= LI + D; i++) g[i + m * SK] = v[i];
#pragma unroll
            for (int j = 1; j <= LJ; j++) {
#pragma unroll
                for (int n = 0; n <= LIJ - j; n++) v[n] = v[n + 1] + ab * v[n];
#pragma unroll
                for (int i = 0; i <= LI + D; i++) g[i + j * SJ + m * SK] = v[i];
            }
        }
        if (m < LKL) {
            double nxt[LIJ + 1];
#pragma unroll
            for (int n = 0; n <= LIJ; n++)
                nxt[n] = c01 * cur[n] + (m ? m * b01 * prev[n] : 0.0) + (n ? n * b00 * cur[n - 1] : 0.0);
#pragma unroll
            for (int n = 0; n <= LIJ; n++) {
                prev[n] = cur[n];
                cur[n] = nxt[n];
            }
        }
    }
    if (LL > 0) {
#pragma unroll
        for (int o = 0; o < SK; o++) {
            double w[LKL + 1];
#pragma unroll
            for (int m = 0; m <= LKL; m++) w[m] = g[o + m * SK];
#pragma unroll
            for (int l = 1; l <= LL; l++) {
#pragma unroll
                for (int m = 0; m <= LKL - l; m++) w[m] = w[m + 1] + cd * w[m];
#pragma unroll
                for (int k = 0; k <= LK; k++) g[o + k * SK + l * SL] = w[k];
            }
        }
    }
}

#define CB_G(c) case c: build_g_fixed<D, (c) / 27, ((c) / 9) % 3, ((c) / 3) % 3, (c) % 3>(p, dir, ab, cd, g); return;
#define CB_G9(b) CB_G(b) CB_G(b + 1) CB_G(b + 2) CB_G(b + 3) CB_G(b + 4) CB_G(b + 5) CB_G(b + 6) CB_G(b + 7) CB_G(b + 8)

template <int D, bool LOW>
__device__ __forceinline__ void build_g_any(const double *__restrict__ p, int dir, int li, int lj, int lk, int ll,
                                            double ab, double cd, double *__restrict__ g)
{
    if (LOW || (li <= 2 && lj <= 2 && lk <= 2 && ll <= 2)) {
        switch (li * 27 + lj * 9 + lk * 3 + ll) {
            CB_G9(0) CB_G9(9) CB_G9(18) CB_G9(27) CB_G9(36) CB_G9(45) CB_G9(54) CB_G9(63) CB_G9(72)
            default: break;
        }
    }
    if (!LOW) build_g<D>(p, dir, li, lj, lk, ll, ab, cd, g);
}
#undef CB_G9
#undef CB_G


// MODE_FULL (int2e over unique quartets): one integral into all eight index
// orders of the dense [n]^4 tensor so.out (repeats for equal shells write the
// same value twice).
__device__ __forceinline__ void full_store8(double *__restrict__ g, long long n, long long i, long long j,
                                            long long k, long long l, double v)
{
    g[((i * n + j) * n + k) * n + l] = v;
    g[((j * n + i) * n + k) * n + l] = v;
    g[((i * n + j) * n + l) * n + k] = v;
    g[((j * n + i) * n + l) * n + k] = v;
    g[((k * n + l) * n + i) * n + j] = v;
    g[((l * n + k) * n + i) * n + j] = v;
    g[((k * n + l) * n + j) * n + i] = v;
    g[((l * n + k) * n + j) * n + i] = v;
}

struct S2klOut {
    double *out;
    long long nao_pair, comp_stride;
    int nao, i_base;
    // spherical s2kl output (c2s set; l <= 2 kernels): cart->sph factors of a
    // d shell, c2s[s * 6 + c] (s and p: identity), and the spherical AO offset
    // of every shell; out, nao, nao_pair, comp_stride and i_base then describe
    // the spherical block
    const double *c2s;
    const int *ao_sph;
    // MODE_GRAD: rows [g_row0, g_row0 + g_rows) of the dense [nao]^4 density in
    // the Cartesian AO basis (all rows: g_row0 = 0, g_rows = nao)
    const double *gamma;
    int g_row0, g_rows;

    // gamma[i][j][k][l]; 0 for a first index outside the rows held
    __device__ __forceinline__ double gamma_at(long long i, long long j, long long k, long long l) const
    {
        const long long r = i - g_row0;
        if (r < 0 || r >= g_rows) return 0.0;
        const long long n = nao;
        return gamma[((r * n + j) * n + k) * n + l];
    }
};

template <int NT>
__device__ __forceinline__ void grp_sync();

// Spherical s2kl epilogue.  The quartet's Cartesian block, staged in shared
// memory as a[c][fi][fj][fk][fl] (shells in the quartet's own order, nc
// components), is transformed one index at a time (l, k, j, i; d shells only,
// the s and p factors are the identity), alternating between a and b (each
// nc * nf doubles), and written to the spherical s2kl block (k >= l within a
// shell pair with ksh == lsh).  bad: the block did not fit the shared-memory
// staging; its outputs are written as NaN so the failure cannot pass silently.
template <int NT>
__device__ void s2kl_sph_store(double *__restrict__ a, double *__restrict__ b, int nc, int li, int lj, int lk,
                               int ll, int ish, int jsh, int ksh, int lsh, const S2klOut &so, int lane, bool bad)
{
    const int L[4] = {li, lj, lk, ll};
    int n[4] = {ncart(li), ncart(lj), ncart(lk), ncart(ll)};
    double *src = a, *dst = b;
    for (int x = 3; x >= 0; x--) {
        if (L[x] < 2 || bad) continue;
        int outer = nc, inner = 1;
        for (int y = 0; y < x; y++) outer *= n[y];
        for (int y = x + 1; y < 4; y++) inner *= n[y];
        const int m = 2 * L[x] + 1, nx = n[x];
        grp_sync<NT>();
        for (int e = lane; e < outer * m * inner; e += NT) {
            const int in = e % inner, t = e / inner;
            const int sidx = t % m, o = t / m;
            const double *sp = src + o * nx * inner + in;
            const double *cr = so.c2s + sidx * 6;
            double v = 0.0;
            for (int c = 0; c < nx; c++) v = fma(cr[c], sp[c * inner], v);
            dst[e] = v;
        }
        n[x] = m;
        double *t = src;
        src = dst;
        dst = t;
    }
    grp_sync<NT>();
    const int i0 = so.ao_sph[ish] - so.i_base, j0 = so.ao_sph[jsh], k0 = so.ao_sph[ksh], l0 = so.ao_sph[lsh];
    const int nl = 2 * ll + 1, nk = 2 * lk + 1, nj = 2 * lj + 1, ni = 2 * li + 1;
    for (int e = lane; e < nc * ni * nj * nk * nl; e += NT) {
        int t = e;
        const int fl = t % nl; t /= nl;
        const int fk = t % nk; t /= nk;
        const int fj = t % nj; t /= nj;
        const int fi = t % ni;
        const int c = t / ni;
        if (ksh == lsh && fl > fk) continue;
        const long long k = k0 + fk, l = l0 + fl;
        so.out[c * so.comp_stride + ((long long)(i0 + fi) * so.nao + (j0 + fj)) * so.nao_pair + k * (k + 1) / 2 + l] =
            bad ? __longlong_as_double(0x7ff8000000000000ll) : src[e];
    }
    grp_sync<NT>();
}

// Integrals of one shell quartet by one warp.  MODE_S2KL writes the s2kl block,
// MODE_QSUM writes two checksums per component of the Cartesian quartet block,
// MODE_GRAD contracts the block with so.gamma: per component
//   q[c] += w * sum_{ijkl in the block} I_c[ijkl] gamma[ijkl],
// w = 1 for k shell == l shell (the full k,l block) and 2 otherwise (the
// (l,k) half of a gamma that is symmetric in k <-> l).
// GW outputs per lane and chunk (eri_quartet_any sizes it to the block).
template <int D, int MODE, bool LOW, int GW = 8>
__device__ void eri_quartet(const int *__restrict__ atm, const int *__restrict__ bas,
                            const double *__restrict__ env, const int *__restrict__ ao_loc,
                            int ish, int jsh, int ksh, int lsh, double *__restrict__ wsm, int smem_warp,
                            const S2klOut &so, double *__restrict__ qsum, int lane)
{
    constexpr int NC = D ? 3 : 1;
    const Shell si = load_shell(atm, bas, env, ish), sj_ = load_shell(atm, bas, env, jsh);
    const Shell sk_ = load_shell(atm, bas, env, ksh), sl_ = load_shell(atm, bas, env, lsh);
    const int li = si.l, lj = sj_.l, lk = sk_.l, ll = sl_.l;
    const int nfi = ncart(li), nfj = ncart(lj), nfk = ncart(lk), nfl = ncart(ll);
    const int nf = nfi * nfj * nfk * nfl;
    const int nroots = (li + lj + lk + ll + D) / 2 + 1;
    const int sj = li + 1 + D, sk = sj * (lj + 1), sl = sk * (lk + 1), gsz = sl * (ll + 1);
    double AB[3], CD[3];
    for (int x = 0; x < 3; x++) {
        AB[x] = si.R[x] - sj_.R[x];
        CD[x] = sk_.R[x] - sl_.R[x];
    }
    const double rab2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    const double rcd2 = CD[0] * CD[0] + CD[1] * CD[1] + CD[2] * CD[2];
    const PairMask mb = pair_mask(si, sj_, rab2, li + lj + D), mk = pair_mask(sk_, sl_, rcd2, lk + ll);
    const int nslot = mb.n * mk.n * nroots;
    const double pref0 = 34.986836655249725693 * common_fac(li) * common_fac(lj) * common_fac(lk) *
                         common_fac(ll);   // 2 pi^(5/2) x angular factors of s, p
    // shared memory: [pair rows][slot parameters][2D tables]
    // per-direction table stride: odd, so the lanes of phase B (one table
    // each) and of phase C (different elements of one table) spread over the banks
    const int gst = gsz | 1;
    int tabn = (mb.n + mk.n) * kPairStride;
    if (!pair_table_fits(tabn, smem_warp, 3 * gst + kParStride, nslot)) tabn = 0;
    int ns = (smem_warp - tabn) / (3 * gst + kParStride);
    ns = ns > kMaxSlots ? kMaxSlots : ns;
    double *tab = tabn ? wsm : nullptr;
    double *par = wsm + tabn;
    double *gbuf = par + ns * kParStride;
    if (tab) build_pair_tables(si, sj_, sk_, sl_, mb, mk, AB, rab2, CD, rcd2, tab, lane, 32);

    // Small blocks: the warp splits into NG slot groups of FW lanes (FW >= nf),
    // each group accumulates a strided subset of the slots, and the groups are
    // reduced with shuffles at the end.  nf >= 32: one group, GW outputs per lane.
    const int FW = nf >= 32 ? 32 : (nf > 16 ? 32 : (nf > 8 ? 16 : (nf > 4 ? 8 : (nf > 2 ? 4 : (nf > 1 ? 2 : 1)))));
    const int NG = 32 / FW;
    const int flane = lane & (FW - 1), grp = lane / FW;
    for (int f0 = 0; f0 < nf; f0 += FW * GW) {
        double acc[GW][NC];
        int gidx[GW];     // ax | ay << 10 | az << 20
        int iexp[D ? GW : 1];     // ix | iy << 4 | iz << 8 (derivative only)
#pragma unroll
        for (int n = 0; n < GW; n++) {
#pragma unroll
            for (int c = 0; c < NC; c++) acc[n][c] = 0.0;
            const int f = f0 + n * FW + flane;
            gidx[n] = 0;
            if (D) iexp[D ? n : 0] = 0;
            if (f < nf) {
                int t = f;
                const int fl = t % nfl; t /= nfl;
                const int fk = t % nfk; t /= nfk;
                const int fj = t % nfj;
                const int fi = t / nfj;
                const int ci = c_cart[c_cart_off[li] + fi], cj = c_cart[c_cart_off[lj] + fj];
                const int ck = c_cart[c_cart_off[lk] + fk], cl = c_cart[c_cart_off[ll] + fl];
                const int ax = (ci & 15) + (cj & 15) * sj + (ck & 15) * sk + (cl & 15) * sl;
                const int ay = ((ci >> 4) & 15) + ((cj >> 4) & 15) * sj + ((ck >> 4) & 15) * sk + ((cl >> 4) & 15) * sl;
                const int az = (ci >> 8) + (cj >> 8) * sj + (ck >> 8) * sk + (cl >> 8) * sl;
                gidx[n] = ax | (ay << 10) | (az << 20);
                if (D) iexp[D ? n : 0] = ci;
            }
        }
        for (int s0 = 0; s0 < nslot; s0 += ns) {
            const int s1 = min(nslot, s0 + ns);
            __syncwarp();
            // ---- phase A: Rys nodes/weights and recurrence coefficients, one slot per lane
            slot_params(tab, si, sj_, sk_, sl_, mb, mk, AB, rab2, CD, rcd2, nroots, pref0, s0, s1, par, lane, 32);
            __syncwarp();
            // ---- phase B: recurrences, one (slot, direction) per lane
            for (int it = lane; it < (s1 - s0) * 3; it += 32) {
                const int s = it / 3, dir = it - s * 3;
                build_g_any<D, LOW>(par + s * kParStride, dir, li, lj, lk, ll, AB[dir], CD[dir],
                                    gbuf + (s * 3 + dir) * gst);
            }
            __syncwarp();
            // ---- phase C: accumulate
            for (int s = grp; s < s1 - s0; s += NG) {
                const double *gx = gbuf + s * 3 * gst, *gy = gx + gst, *gz = gy + gst;
                const double ai2 = par[s * kParStride + 10];
#pragma unroll
                for (int n = 0; n < GW; n++) {
                    if (f0 + n * FW + flane < nf) {
                        const int ax = gidx[n] & 1023, ay = (gidx[n] >> 10) & 1023, az = gidx[n] >> 20;
                        const double x = gx[ax], y = gy[ay], z = gz[az];
                        if (D == 0) {
                            acc[n][0] = fma(x * y, z, acc[n][0]);
                        } else {
                            const int ie = iexp[D ? n : 0];
                            const int ix = ie & 15, iy = (ie >> 4) & 15, iz = ie >> 8;
                            double fx = -ai2 * gx[ax + 1], fy = -ai2 * gy[ay + 1], fz = -ai2 * gz[az + 1];
                            if (ix) fx = fma((double)ix, gx[ax - 1], fx);
                            if (iy) fy = fma((double)iy, gy[ay - 1], fy);
                            if (iz) fz = fma((double)iz, gz[az - 1], fz);
                            acc[n][0] = fma(fx * y, z, acc[n][0]);
                            acc[n][NC > 1 ? 1 : 0] = fma(x * fy, z, acc[n][NC > 1 ? 1 : 0]);
                            acc[n][NC > 2 ? 2 : 0] = fma(x * y, fz, acc[n][NC > 2 ? 2 : 0]);
                        }
                    }
                }
            }
        }
        // ---- reduce the slot groups
        if (NG > 1) {
#pragma unroll
            for (int n = 0; n < GW; n++)
#pragma unroll
                for (int c = 0; c < NC; c++)
                    for (int o = FW; o < 32; o <<= 1) acc[n][c] += __shfl_xor_sync(0xffffffffu, acc[n][c], o);
        }
        // ---- epilogue
        if (MODE == MODE_S2KL_SPH) {
            // spherical output: the block (one chunk of at most FW * GW
            // functions on this path) is staged over the dead slot buffers
            __syncwarp();
            const bool bad = nf > FW * GW || 2 * NC * nf > smem_warp;
            double *a = wsm, *b = wsm + NC * nf;
            if (!bad) {
#pragma unroll
                for (int n = 0; n < GW; n++) {
                    const int f = f0 + n * FW + flane;
                    if (f < nf && grp == 0)
#pragma unroll
                        for (int c = 0; c < NC; c++) a[c * nf + f] = acc[n][c];
                }
            }
            s2kl_sph_store<32>(a, b, NC, li, lj, lk, ll, ish, jsh, ksh, lsh, so, lane, bad);
        } else if (MODE == MODE_S2KL) {
            const int i0 = ao_loc[ish] - so.i_base, j0 = ao_loc[jsh], k0 = ao_loc[ksh], l0 = ao_loc[lsh];
#pragma unroll
            for (int n = 0; n < GW; n++) {
                const int f = f0 + n * FW + flane;
                if (f < nf && grp == 0) {
                    int t = f;
                    const int fl = t % nfl; t /= nfl;
                    const int fk = t % nfk; t /= nfk;
                    const int fj = t % nfj;
                    const int fi = t / nfj;
                    if (ksh == lsh && fl > fk) continue;
                    const long long k = k0 + fk, l = l0 + fl;
                    const long long addr = ((long long)(i0 + fi) * so.nao + (j0 + fj)) * so.nao_pair + k * (k + 1) / 2 + l;
#pragma unroll
                    for (int c = 0; c < NC; c++) so.out[c * so.comp_stride + addr] = acc[n][c];
                }
            }
        } else if (MODE == MODE_FULL) {
            const int i0 = ao_loc[ish], j0 = ao_loc[jsh], k0 = ao_loc[ksh], l0 = ao_loc[lsh];
#pragma unroll
            for (int n = 0; n < GW; n++) {
                const int f = f0 + n * FW + flane;
                if (f < nf && grp == 0) {
                    int t = f;
                    const int fl = t % nfl; t /= nfl;
                    const int fk = t % nfk; t /= nfk;
                    const int fj = t % nfj;
                    const int fi = t / nfj;
                    full_store8(so.out, so.nao, i0 + fi, j0 + fj, k0 + fk, l0 + fl, acc[n][0]);
                }
            }
        } else if (MODE == MODE_GRAD) {
            const long long nao = so.nao;
            const int i0 = ao_loc[ish], j0 = ao_loc[jsh], k0 = ao_loc[ksh], l0 = ao_loc[lsh];
            double sv[NC];
#pragma unroll
            for (int c = 0; c < NC; c++) sv[c] = 0.0;
#pragma unroll
            for (int n = 0; n < GW; n++) {
                const int f = f0 + n * FW + flane;
                if (f < nf && grp == 0) {
                    int t = f;
                    const int fl = t % nfl; t /= nfl;
                    const int fk = t % nfk; t /= nfk;
                    const int fj = t % nfj;
                    const int fi = t / nfj;
                    const double gv = so.gamma_at(i0 + fi, j0 + fj, k0 + fk, l0 + fl);
#pragma unroll
                    for (int c = 0; c < NC; c++) sv[c] = fma(acc[n][c], gv, sv[c]);
                }
            }
            const double wkl = ksh == lsh ? 1.0 : 2.0;
#pragma unroll
            for (int c = 0; c < NC; c++) {
                for (int o = 16; o > 0; o >>= 1) sv[c] += __shfl_xor_sync(0xffffffffu, sv[c], o);
                if (lane == 0) qsum[c] += wkl * sv[c];
            }
        } else {
#pragma unroll
            for (int c = 0; c < NC; c++) {
                double s1v = 0.0, s2v = 0.0;
#pragma unroll
                for (int n = 0; n < GW; n++) {
                    const int f = f0 + n * FW + flane;
                    if (f < nf && grp == 0) {
                        s1v += acc[n][c] * (1.0 + 0.125 * (f & 7));
                        s2v += acc[n][c] * acc[n][c];
                    }
                }
                for (int o = 16; o > 0; o >>= 1) {
                    s1v += __shfl_xor_sync(0xffffffffu, s1v, o);
                    s2v += __shfl_xor_sync(0xffffffffu, s2v, o);
                }
                if (lane == 0) {
                    qsum[2 * c] += s1v;
                    qsum[2 * c + 1] += s2v;
                }
            }
        }
    }
}

// The per-output path with GW sized to the block: every lane holds at most
// ceil(nf / FW) outputs (FW lanes per slot group), so the unrolled output
// loop of the slot accumulation has no iterations that no lane uses; blocks
// of more than 8 FW functions run in chunks of 8 per lane.
template <int D, int MODE, bool LOW>
__device__ __forceinline__ void eri_quartet_any(const int *__restrict__ atm, const int *__restrict__ bas,
                                                const double *__restrict__ env, const int *__restrict__ ao_loc,
                                                int ish, int jsh, int ksh, int lsh, double *__restrict__ wsm,
                                                int smem_warp, const S2klOut &so, double *__restrict__ qsum,
                                                int lane, int nf)
{
    const int fw = nf >= 32 ? 32 : (nf > 16 ? 32 : (nf > 8 ? 16 : (nf > 4 ? 8 : (nf > 2 ? 4 : (nf > 1 ? 2 : 1)))));
    const int per = (nf + fw - 1) / fw;
    if (per <= 1)
        eri_quartet<D, MODE, LOW, 1>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, wsm, smem_warp, so, qsum, lane);
    else if (per <= 2)
        eri_quartet<D, MODE, LOW, 2>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, wsm, smem_warp, so, qsum, lane);
    else if (per <= 4)
        eri_quartet<D, MODE, LOW, 4>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, wsm, smem_warp, so, qsum, lane);
    else
        eri_quartet<D, MODE, LOW, 8>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, wsm, smem_warp, so, qsum, lane);
}

// ===========================================================================
// Contracted-HRR path for l <= 2 quartets (one warp per quartet).
//
// The warp path above applies both horizontal recurrences (HRR) to the 2D
// tables of every slot and forms every output of the block per slot.  For
// contracted shells (many primitive quartets x roots) it is cheaper to
// accumulate the vertical/transfer-recurrence integrals
//     [e|f] = sum_slots Ix(ex,fx) Iy(ey,fy) Iz(ez,fz),  |e| = A0..A0+lj,
//                                                       |f| = lk..lk+ll,
// over all slots (registers, lane-owned) and to run the HRR once, in 6D, on
// the contracted [e|f]:
//     (e|c, d+1_x) = (e|c+1_x, d) + CD_x (e|c, d)        (ket, per e row)
//     (a, b+1_x|   = (a+1_x, b|   + AB_x (a, b|         (bra, per (c,d) column)
// int2e uses one set with A0 = li.  int2e_ip1 uses two: A0 = li + 1 with the
// factor 2 a_i folded into each slot, and A0 = li - 1; the derivative is
//     d/dx_i (ij|kl) = i_x (i-1_x j|kl) - 2 a_i (i+1_x j|kl).
// Per slot this is 3 loads + 3 flops per [e|f] value instead of ~9 loads and
// ~15 flops per output and component, and the recurrences run once per batch
// instead of once per 256-output chunk.
// ===========================================================================
static constexpr int kHcMaxJ = 40;      // accumulators per lane (<= 1280 per quartet)

__host__ __device__ constexpr int hc_ncart(int l) { return (l + 1) * (l + 2) / 2; }
__host__ __device__ constexpr int hc_csum(int l0, int l1)
{
    int s = 0;
    for (int l = l0; l <= l1; l++) s += hc_ncart(l);
    return s;
}
// Cartesian component k of shell l (order xx, xy, xz, yy, yz, zz, ...)
__host__ __device__ constexpr int hc_n(int k)
{
    int n = 0;
    while ((n + 1) * (n + 2) / 2 <= k) n++;
    return n;
}
__host__ __device__ constexpr int hc_lx(int l, int k) { return l - hc_n(k); }
__host__ __device__ constexpr int hc_lz(int k) { return k - hc_n(k) * (hc_n(k) + 1) / 2; }
__host__ __device__ constexpr int hc_ly(int l, int k) { return hc_n(k) - hc_lz(k); }
__host__ __device__ constexpr int hc_idx(int lx, int ly, int lz) { return (ly + lz) * (ly + lz + 1) / 2 + lz; }
// index in shell l+1 of component k of shell l raised by one in direction x
__host__ __device__ constexpr int hc_up(int l, int k, int x)
{
    return hc_idx(hc_lx(l, k) + (x == 0), hc_ly(l, k) + (x == 1), hc_lz(k) + (x == 2));
}

// 2D vertical + transfer recurrences of one (slot, direction), no HRR:
// g[e + f * (LE + 1)], e <= LE, f <= LF.
template <int LE, int LF>
__device__ __noinline__ void hc_build_2d(const double *__restrict__ p, int dir, double *__restrict__ g)
{
    const double c00 = p[dir], c01 = p[3 + dir], b00 = p[6], b10 = p[7], b01 = p[8];
    double prev[LE + 1], cur[LE + 1];
    cur[0] = dir == 0 ? p[9] : 1.0;
#pragma unroll
    for (int n = 0; n < LE; n++) cur[n + 1] = c00 * cur[n] + (n ? n * b10 * cur[n - 1] : 0.0);
#pragma unroll
    for (int n = 0; n <= LE; n++) prev[n] = 0.0;
#pragma unroll
    for (int m = 0; m <= LF; m++) {
#pragma unroll
        for (int n = 0; n <= LE; n++) g[n + m * (LE + 1)] = cur[n];
        if (m < LF) {
            double nxt[LE + 1];
#pragma unroll
            for (int n = 0; n <= LE; n++)
                nxt[n] = c01 * cur[n] + (m ? m * b01 * prev[n] : 0.0) + (n ? n * b00 * cur[n - 1] : 0.0);
#pragma unroll
            for (int n = 0; n <= LE; n++) {
                prev[n] = cur[n];
                cur[n] = nxt[n];
            }
        }
    }
}

#define CB_B2(c) case c: hc_build_2d<(c) / 5, (c) % 5>(p, dir, g); return;
__device__ __forceinline__ void hc_build_any(const double *__restrict__ p, int dir, int le, int lf,
                                             double *__restrict__ g)
{
    switch (le * 5 + lf) {
        CB_B2(0) CB_B2(1) CB_B2(2) CB_B2(3) CB_B2(4) CB_B2(5) CB_B2(6) CB_B2(7) CB_B2(8) CB_B2(9)
        CB_B2(10) CB_B2(11) CB_B2(12) CB_B2(13) CB_B2(14) CB_B2(15) CB_B2(16) CB_B2(17) CB_B2(18) CB_B2(19)
        CB_B2(20) CB_B2(21) CB_B2(22) CB_B2(23) CB_B2(24) CB_B2(25) CB_B2(26) CB_B2(27) CB_B2(28) CB_B2(29)
        default: break;
    }
}
#undef CB_B2

// One line of the 6D HRR in registers: in[s * istride], s over the components
// of shells L0..L0+L1 (shell-major), -> out[(a * ncart(L1) + b) * ostride],
// (a, b+1_x) = (a+1_x, b) + R_x (a, b).  L1 <= 2.
template <int L0, int L1>
__device__ __noinline__ void hc_hrr_line(const double *__restrict__ in, int istride, double *__restrict__ out,
                                         int ostride, double rx, double ry, double rz)
{
    constexpr int N0 = hc_csum(L0, L0 + L1);
    constexpr int NA = hc_ncart(L0);
    double v0[N0];
#pragma unroll
    for (int s = 0; s < N0; s++) v0[s] = in[s * istride];
    if constexpr (L1 == 0) {
#pragma unroll
        for (int a = 0; a < NA; a++) out[a * ostride] = v0[a];
    } else {
        const double R[3] = {rx, ry, rz};
        // level 1: (a, 1_x) for |a| = L0 .. L0+L1-1, stored v1[x][a-flat]
        constexpr int N1 = hc_csum(L0, L0 + L1 - 1);
        double v1[3][N1];
#pragma unroll
        for (int x = 0; x < 3; x++) {
            int off = 0, offu = NA;        // start of shell A (flat) and of shell A+1 in v0
#pragma unroll
            for (int A = L0; A < L0 + L1; A++) {
#pragma unroll
                for (int k = 0; k < hc_ncart(A); k++)
                    v1[x][off + k] = v0[offu + hc_up(A, k, x)] + R[x] * v0[off + k];
                off += hc_ncart(A);
                offu += hc_ncart(A + 1);
            }
        }
        if constexpr (L1 == 1) {
#pragma unroll
            for (int a = 0; a < NA; a++)
#pragma unroll
                for (int x = 0; x < 3; x++) out[(a * 3 + x) * ostride] = v1[x][a];
        } else {
            // level 2: b in (xx, xy, xz, yy, yz, zz); first raised direction x,
            // b - 1_x in level 1 as direction y
            constexpr int bx[6] = {0, 0, 0, 1, 1, 2};     // direction peeled off
            constexpr int by[6] = {0, 1, 2, 1, 2, 2};     // level-1 direction left
#pragma unroll
            for (int a = 0; a < NA; a++)
#pragma unroll
                for (int b = 0; b < 6; b++)
                    out[(a * 6 + b) * ostride] = v1[by[b]][NA + hc_up(L0, a, bx[b])] + R[bx[b]] * v1[by[b]][a];
        }
    }
}

#define CB_H(c) case c: hc_hrr_line<(c) / 3, (c) % 3>(in, istride, out, ostride, rx, ry, rz); return;
__device__ __forceinline__ void hc_hrr_any(int l0, int l1, const double *__restrict__ in, int istride,
                                           double *__restrict__ out, int ostride, double rx, double ry, double rz)
{
    switch (l0 * 3 + l1) {
        CB_H(0) CB_H(1) CB_H(2) CB_H(3) CB_H(4) CB_H(5) CB_H(6) CB_H(7) CB_H(8) CB_H(9) CB_H(10) CB_H(11)
        default: break;
    }
}
#undef CB_H

// Layout of one quartet on this path; hc_plan() decides whether it applies.
// The quartet may be computed as (ij|lk) (kswap: the larger ket shell carries
// the recurrences) or, for int2e, as (ji|kl) (bswap); outputs are mapped back.
struct HcPlan {
    int nset, a0[2], ne[2], nf_ket, nacc, setoff[2];
    int nc, nd, ncd, na[2], nb, rowoff[2], nrows, braoff[2], nbra, nket;
    // grouped accumulation: groups (set, ex, ey, ket component f), members
    // ez = ez_lo .. ez_lo + ze - 1 (ze = lj + 1); gset0 groups in set 0
    int ngrp, gset0, ze;
    bool kswap, bswap;
};

static constexpr int kHcMaxG = 8;       // groups per lane on a warp (grouped form)

// force: 0 the measured rule below, 1 this path whenever the quartet fits,
// 2 never (the per-output path); the warp kernels take it per L-class from
// the autotuner's table (PathTable).
__device__ __forceinline__ bool hc_plan(int D, int li, int lj, int lk, int ll, HcPlan &h,
                                        int maxacc = 32 * kHcMaxJ, int cap = kHcSmem, bool always = false,
                                        int force = 0)
{
    if (li > 2 || lj > 2 || lk > 2 || ll > 2 || force == 2) return false;
    h.kswap = lk < ll;
    h.bswap = D == 0 && li < lj;
    if (h.kswap) { const int t = lk; lk = ll; ll = t; }
    if (h.bswap) { const int t = li; li = lj; lj = t; }
    h.nset = D ? (li > 0 ? 2 : 1) : 1;
    h.a0[0] = D ? li + 1 : li;
    h.a0[1] = li - 1;
    h.nf_ket = hc_csum(lk, lk + ll);
    h.nc = hc_ncart(lk);
    h.nd = hc_ncart(ll);
    h.ncd = h.nc * h.nd;
    h.nb = hc_ncart(lj);
    h.nacc = 0;
    h.nrows = 0;
    h.nbra = 0;
    for (int s = 0; s < h.nset; s++) {
        h.ne[s] = hc_csum(h.a0[s], h.a0[s] + lj);
        h.na[s] = hc_ncart(h.a0[s]);
        h.setoff[s] = h.nacc;
        h.nacc += h.ne[s] * h.nf_ket;
        h.rowoff[s] = h.nrows;
        h.nrows += h.ne[s];
        h.braoff[s] = h.nbra;
        h.nbra += h.na[s] * h.nb;
    }
    h.nket = h.nrows * h.ncd;
    h.ze = lj + 1;
    h.gset0 = 0;
    h.ngrp = 0;
    for (int s = 0; s < h.nset; s++) {
        const int m = h.a0[s] + lj;           // largest |e| of the set
        const int g = (m + 1) * (m + 2) / 2 * h.nf_ket;
        if (s == 0) h.gset0 = g;
        h.ngrp += g;
    }
    const int nf = hc_ncart(li) * h.nb * h.ncd;
    const int lo = h.nacc > h.nbra * h.ncd ? h.nacc : h.nbra * h.ncd;
    if (h.nacc > maxacc || lo + h.nket > cap) return false;
    if (always || force == 1) return true;
    // measured: worth it when the per-output path would recompute the slots
    // for several 256-output chunks, or when [e|f] is clearly smaller than
    // the output block and the ket has no s shell
    return nf > 256 || (ll > 0 && 100 * h.nacc <= 62 * nf * (D ? 3 : 1));
}

template <int NT>
__device__ __forceinline__ void grp_sync()
{
    if (NT == 32) __syncwarp();
    else __syncthreads();
}

// Sum of ncart(l) for l = 0..n (tetrahedral numbers; 0 for n = -1).
__host__ __device__ constexpr int hc_tet(int n) { return (n + 1) * (n + 2) * (n + 3) / 6; }

// Group t of the grouped accumulation: set s, bra exponents ex, ey, members
// ez = ezlo .. ezlo + nm - 1 (every |e| = ex + ey + ez in [a0[s], a0[s] + lj]),
// ket component jf of shell F and its flat ket index ff (shells lk.. in order).
__device__ __forceinline__ void hc_group(const HcPlan &h, int lj, int lk, int t, int &s, int &ex, int &ey,
                                         int &ezlo, int &nm, int &F, int &jf, int &ff)
{
    s = (h.nset > 1 && t >= h.gset0) ? 1 : 0;
    const int r = t - (s ? h.gset0 : 0);
    int pe = r / h.nf_ket;
    ff = r - pe * h.nf_ket;
    const int m = h.a0[s] + lj;
    ex = 0;
    while (pe > m - ex) {
        pe -= m - ex + 1;
        ex++;
    }
    ey = pe;
    ezlo = h.a0[s] - ex - ey > 0 ? h.a0[s] - ex - ey : 0;
    nm = m - ex - ey - ezlo + 1;
    jf = ff;
    F = lk;
    while (jf >= hc_ncart(F)) {
        jf -= hc_ncart(F);
        F++;
    }
}

// NT cooperating threads (a warp, or a 256-thread CTA for heavy quartets),
// `cap` doubles of shared memory at wsm; `qsum` is added to (warp) or
// assigned (CTA) in the checksum and gradient modes.
//
// ZE = 0: each lane owns NJ [e|f] accumulators (3 shared-memory loads per
// value and slot).  ZE > 0 (grouped): each lane owns NJ groups; a group is one
// (set, ex, ey, ket component f) and its members run over ez (at most ZE = lj
// + 1 of them), so they share the product Ix(ex, fx) Iy(ey, fy) and read
// consecutive Iz entries: 2 + (members) loads per group and slot.
template <int D, int MODE, int NJ, int NT, int ZE = 0>
__device__ void eri_quartet_hc(const int *__restrict__ atm, const int *__restrict__ bas,
                               const double *__restrict__ env, const int *__restrict__ ao_loc, int ish, int jsh,
                               int ksh, int lsh, const HcPlan &h, double *__restrict__ wsm, const S2klOut &so,
                               double *__restrict__ qsum, int lane, int cap)
{
    constexpr int NC = D ? 3 : 1;
    constexpr int NM = ZE ? ZE : 1;
    const Shell si = load_shell(atm, bas, env, h.bswap ? jsh : ish), sj_ = load_shell(atm, bas, env, h.bswap ? ish : jsh);
    const Shell sk_ = load_shell(atm, bas, env, h.kswap ? lsh : ksh), sl_ = load_shell(atm, bas, env, h.kswap ? ksh : lsh);
    const int li = si.l, lj = sj_.l, lk = sk_.l, ll = sl_.l;      // computed orientation
    const int le = li + lj + D, lf = lk + ll, s2 = (le + 1) * (lf + 1);
    const int nroots = (li + lj + lk + ll + D) / 2 + 1;
    double AB[3], CD[3];
    for (int x = 0; x < 3; x++) {
        AB[x] = si.R[x] - sj_.R[x];
        CD[x] = sk_.R[x] - sl_.R[x];
    }
    const double rab2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    const double rcd2 = CD[0] * CD[0] + CD[1] * CD[1] + CD[2] * CD[2];
    const PairMask mb = pair_mask(si, sj_, rab2, li + lj + D), mk = pair_mask(sk_, sl_, rcd2, lk + ll);
    const int nslot = mb.n * mk.n * nroots;
    const double pref0 = 34.986836655249725693 * common_fac(li) * common_fac(lj) * common_fac(lk) *
                         common_fac(ll);
    // shared memory: [pair rows][slot parameters][2D tables]
    const int s2t = s2 | 1;     // odd per-direction table stride (bank spread)
    int tabn = (mb.n + mk.n) * kPairStride;
    if (!pair_table_fits(tabn, cap, 3 * s2t + kParStride, nslot)) tabn = 0;
    int ns = (cap - tabn) / (3 * s2t + kParStride);
    ns = ns > (NT > 32 ? kMaxSlotsCta : kMaxSlots) ? (NT > 32 ? kMaxSlotsCta : kMaxSlots) : ns;
    double *tab = tabn ? wsm : nullptr;
    double *par = wsm + tabn;
    double *gbuf = par + ns * kParStride;
    if (tab) build_pair_tables(si, sj_, sk_, sl_, mb, mk, AB, rab2, CD, rcd2, tab, lane, NT);

    // ZE = 0: lane-owned accumulators, flat t = lane + NT j = setoff[s] + ie * nf_ket + if,
    //         idx[j] = x | y << 8 | z << 16 (table offsets) | raised set << 24;
    // ZE > 0: lane-owned groups t = lane + NT j,
    //         idx[j] = x | y << 8 | z(ezlo) << 16 | (members - 1) << 24 | raised set << 26
    const int se = le + 1;
    int idx[NJ];
    double acc[NJ][NM];
    const int nj = ((ZE ? h.ngrp : h.nacc) - lane + NT - 1) / NT;
#pragma unroll
    for (int j = 0; j < NJ; j++) {
#pragma unroll
        for (int m = 0; m < NM; m++) acc[j][m] = 0.0;
        idx[j] = 0;
        const int t = lane + NT * j;
        if (j < nj) {
            if (ZE) {
                int s, ex, ey, ezlo, nm, F, jf, ff;
                hc_group(h, lj, lk, t, s, ex, ey, ezlo, nm, F, jf, ff);
                const int fx = hc_lx(F, jf), fy = hc_ly(F, jf), fz = hc_lz(jf);
                idx[j] = (ex + fx * se) | ((ey + fy * se) << 8) | ((ezlo + fz * se) << 16) | ((nm - 1) << 24) |
                         ((D && s == 0) ? (1 << 26) : 0);
            } else {
                const int s = (h.nset > 1 && t >= h.setoff[1]) ? 1 : 0;
                const int r = t - h.setoff[s];
                int ie = r / h.nf_ket, jf = r - ie * h.nf_ket;
                int E = h.a0[s];
                while (ie >= hc_ncart(E)) { ie -= hc_ncart(E); E++; }
                int F = lk;
                while (jf >= hc_ncart(F)) { jf -= hc_ncart(F); F++; }
                const int ex = hc_lx(E, ie), ey = hc_ly(E, ie), ez = hc_lz(ie);
                const int fx = hc_lx(F, jf), fy = hc_ly(F, jf), fz = hc_lz(jf);
                idx[j] = (ex + fx * se) | ((ey + fy * se) << 8) | ((ez + fz * se) << 16) |
                         ((D && s == 0) ? (1 << 24) : 0);
            }
        }
    }
    for (int s0 = 0; s0 < nslot; s0 += ns) {
        const int s1 = min(nslot, s0 + ns);
        grp_sync<NT>();
        // ---- phase A: Rys nodes/weights and recurrence coefficients, one slot per thread
        slot_params(tab, si, sj_, sk_, sl_, mb, mk, AB, rab2, CD, rcd2, nroots, pref0, s0, s1, par, lane, NT);
        grp_sync<NT>();
        // ---- phase B: 2D tables, one (slot, direction) per lane
        for (int it = lane; it < (s1 - s0) * 3; it += NT) {
            const int s = it / 3, dir = it - s * 3;
            hc_build_any(par + s * kParStride, dir, le, lf, gbuf + (s * 3 + dir) * s2t);
        }
        grp_sync<NT>();
        // ---- phase C: [e|f] += Ix Iy Iz (x 2 a_i on the raised set)
        for (int s = 0; s < s1 - s0; s++) {
            const double *gx = gbuf + s * 3 * s2t, *gy = gx + s2t, *gz = gy + s2t;
            const double a2 = par[s * kParStride + 10];
#pragma unroll
            for (int j = 0; j < NJ; j++) {
                if (j < nj) {
                    const int o = idx[j];
                    if (ZE) {
                        double v = gx[o & 255] * gy[(o >> 8) & 255];
                        if (D) v *= ((o >> 26) & 1) ? a2 : 1.0;
                        const double *zp = gz + ((o >> 16) & 255);
                        const int nm1 = (o >> 24) & 3;
#pragma unroll
                        for (int m = 0; m < NM; m++)
                            if (m <= nm1) acc[j][m] = fma(v, zp[m], acc[j][m]);
                    } else {
                        const double v = gx[o & 255] * gy[(o >> 8) & 255];
                        acc[j][0] = fma(v * gz[(o >> 16) & 255], (o >> 24) ? a2 : 1.0, acc[j][0]);
                    }
                }
            }
        }
    }
    // ---- contracted HRR.  Shared memory: [e|f] at [0, nacc), ket rows at the
    // top [cap - nket, cap), bra results at [0, nbra * ncd).
    grp_sync<NT>();
#pragma unroll
    for (int j = 0; j < NJ; j++) {
        if (j < nj) {
            if (ZE) {
                int s, ex, ey, ezlo, nm, F, jf, ff;
                hc_group(h, lj, lk, lane + NT * j, s, ex, ey, ezlo, nm, F, jf, ff);
                const int base = h.setoff[s] + ff, t0 = hc_tet(h.a0[s] - 1);
#pragma unroll
                for (int m = 0; m < NM; m++) {
                    if (m < nm) {
                        const int ez = ezlo + m;
                        const int ie = hc_tet(ex + ey + ez - 1) - t0 + hc_idx(ex, ey, ez);
                        wsm[base + ie * h.nf_ket] = acc[j][m];
                    }
                }
            } else {
                wsm[lane + NT * j] = acc[j][0];
            }
        }
    }
    grp_sync<NT>();
    double *ket = wsm + (cap - h.nket);
    for (int row = lane; row < h.nrows; row += NT) {
        const int s = (h.nset > 1 && row >= h.rowoff[1]) ? 1 : 0;
        const int ie = row - h.rowoff[s];
        hc_hrr_any(lk, ll, wsm + h.setoff[s] + ie * h.nf_ket, 1, ket + row * h.ncd, 1, CD[0], CD[1], CD[2]);
    }
    grp_sync<NT>();
    double *bra = wsm;
    for (int col = lane; col < h.nset * h.ncd; col += NT) {
        const int s = col / h.ncd, cd = col - s * h.ncd;
        hc_hrr_any(h.a0[s], lj, ket + h.rowoff[s] * h.ncd + cd, h.ncd, bra + h.braoff[s] * h.ncd + cd, h.ncd,
                   AB[0], AB[1], AB[2]);
    }
    grp_sync<NT>();
    // ---- outputs (fi, fj, fk, fl) x component, then the MODE epilogue
    const int nfi = hc_ncart(li), nfj = h.nb, nfk = h.nc, nfl = h.nd;      // computed orientation
    const int nf = nfi * nfj * h.ncd;
    const int onj = h.bswap ? nfi : nfj, onk = h.kswap ? nfl : nfk, onl = h.kswap ? nfk : nfl;   // original
    // spherical s2kl output: the block is staged above the bra results
    // (the [e|f] values and ket rows are dead by now)
    const int slo = h.nacc > h.nbra * h.ncd ? h.nacc : h.nbra * h.ncd;
    const bool sph = MODE == MODE_S2KL_SPH;
    const bool sbad = sph && slo + 2 * NC * nf > cap;
    double *sa = wsm + slo, *sb = sa + NC * nf;
    double r1[NC], r2[NC];
#pragma unroll
    for (int c = 0; c < NC; c++) r1[c] = r2[c] = 0.0;
    for (int f = lane; f < nf; f += NT) {
        const int cd = f % h.ncd;
        const int fij = f / h.ncd;
        const int fj = fij % nfj, fi = fij / nfj;
        double v[NC];
        if (D == 0) {
            v[0] = bra[(fi * nfj + fj) * h.ncd + cd];
        } else {
            const int ix = hc_lx(li, fi), iy = hc_ly(li, fi), iz = hc_lz(fi);
            const int ie[3] = {ix, iy, iz};
#pragma unroll
            for (int x = 0; x < NC; x++) {
                const int up = hc_up(li, fi, x);
                double t = -bra[(h.braoff[0] + up * nfj + fj) * h.ncd + cd];
                if (ie[x] > 0) {
                    const int dn = hc_idx(ix - (x == 0), iy - (x == 1), iz - (x == 2));
                    t = fma((double)ie[x], bra[(h.braoff[1] + dn * nfj + fj) * h.ncd + cd], t);
                }
                v[x] = t;
            }
        }
        // back to the original shell order
        int fk = cd / nfl, fl = cd - fk * nfl;
        if (h.kswap) { const int t = fk; fk = fl; fl = t; }
        const int oi = h.bswap ? fj : fi, oj = h.bswap ? fi : fj;
        if (MODE == MODE_S2KL_SPH) {
            const int fr = ((oi * onj + oj) * onk + fk) * onl + fl;
            if (!sbad)
#pragma unroll
                for (int c = 0; c < NC; c++) sa[c * nf + fr] = v[c];
        } else if (MODE == MODE_S2KL) {
            if (ksh == lsh && fl > fk) continue;
            const int i0 = ao_loc[ish] - so.i_base, j0 = ao_loc[jsh], k0 = ao_loc[ksh], l0 = ao_loc[lsh];
            const long long k = k0 + fk, l = l0 + fl;
            const long long addr = ((long long)(i0 + oi) * so.nao + (j0 + oj)) * so.nao_pair + k * (k + 1) / 2 + l;
#pragma unroll
            for (int c = 0; c < NC; c++) so.out[c * so.comp_stride + addr] = v[c];
        } else if (MODE == MODE_FULL) {
            full_store8(so.out, so.nao, ao_loc[ish] + oi, ao_loc[jsh] + oj, ao_loc[ksh] + fk, ao_loc[lsh] + fl, v[0]);
        } else if (MODE == MODE_GRAD) {
            const long long nao = so.nao;
            const int i0 = ao_loc[ish], j0 = ao_loc[jsh], k0 = ao_loc[ksh], l0 = ao_loc[lsh];
            const double gv = so.gamma_at(i0 + oi, j0 + oj, k0 + fk, l0 + fl);
#pragma unroll
            for (int c = 0; c < NC; c++) r1[c] = fma(v[c], gv, r1[c]);
        } else {
            // checksum weights follow the original (fi, fj, fk, fl) row-major function index
            const int fr = ((oi * onj + oj) * onk + fk) * onl + fl;
#pragma unroll
            for (int c = 0; c < NC; c++) {
                r1[c] += v[c] * (1.0 + 0.125 * (fr & 7));
                r2[c] += v[c] * v[c];
            }
        }
    }
    if (sph) {
        grp_sync<NT>();
        s2kl_sph_store<NT>(sa, sb, NC, h.bswap ? lj : li, h.bswap ? li : lj, h.kswap ? ll : lk, h.kswap ? lk : ll,
                           ish, jsh, ksh, lsh, so, lane, sbad);
    }
    if (MODE == MODE_QSUM || MODE == MODE_GRAD) {
        const double wkl = MODE == MODE_GRAD && ksh != lsh ? 2.0 : 1.0;
#pragma unroll
        for (int c = 0; c < NC; c++)
            for (int o = 16; o > 0; o >>= 1) {
                r1[c] += __shfl_xor_sync(0xffffffffu, r1[c], o);
                r2[c] += __shfl_xor_sync(0xffffffffu, r2[c], o);
            }
        if (NT == 32) {
            if (lane == 0)
#pragma unroll
                for (int c = 0; c < NC; c++) {
                    if (MODE == MODE_GRAD) {
                        qsum[c] += wkl * r1[c];
                    } else {
                        qsum[2 * c] += r1[c];
                        qsum[2 * c + 1] += r2[c];
                    }
                }
        } else {
            // CTA: per-warp partials through shared memory, fixed-order sum
            __syncthreads();
            double *red = wsm;
            if ((lane & 31) == 0)
#pragma unroll
                for (int c = 0; c < NC; c++) {
                    red[(lane >> 5) * 6 + 2 * c] = r1[c];
                    red[(lane >> 5) * 6 + 2 * c + 1] = r2[c];
                }
            __syncthreads();
            if (lane == 0)
#pragma unroll
                for (int c = 0; c < NC; c++) {
                    double a = 0.0, b = 0.0;
                    for (int w = 0; w < NT / 32; w++) {
                        a += red[w * 6 + 2 * c];
                        b += red[w * 6 + 2 * c + 1];
                    }
                    if (MODE == MODE_GRAD) {
                        qsum[c] = wkl * a;
                    } else {
                        qsum[2 * c] = a;
                        qsum[2 * c + 1] = b;
                    }
                }
            __syncthreads();
        }
    }
}

// Grouped form: dispatch on the groups per thread (1, 2, 4 or kHcMaxG).
template <int D, int MODE, int NT, int ZE>
__device__ __forceinline__ void eri_quartet_hcg(const int *__restrict__ atm, const int *__restrict__ bas,
                                                const double *__restrict__ env, const int *__restrict__ ao_loc,
                                                int ish, int jsh, int ksh, int lsh, const HcPlan &h,
                                                double *__restrict__ wsm, const S2klOut &so,
                                                double *__restrict__ qsum, int lane, int cap, int ng)
{
    if (ng <= 1)
        eri_quartet_hc<D, MODE, 1, NT, ZE>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, wsm, so, qsum, lane, cap);
    else if (ng <= 2)
        eri_quartet_hc<D, MODE, 2, NT, ZE>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, wsm, so, qsum, lane, cap);
    else if (ng <= 4 || NT > 32)
        eri_quartet_hc<D, MODE, 4, NT, ZE>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, wsm, so, qsum, lane, cap);
    else
        eri_quartet_hc<D, MODE, kHcMaxG, NT, ZE>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, wsm, so, qsum, lane,
                                                 cap);
}

// Dispatch on the accumulator capacity per thread, so the unrolled per-slot
// loop carries no predicated-off iterations beyond the next multiple of 8.
template <int D, int MODE>
__device__ __forceinline__ void eri_quartet_hc_any(const int *__restrict__ atm, const int *__restrict__ bas,
                                                   const double *__restrict__ env, const int *__restrict__ ao_loc,
                                                   int ish, int jsh, int ksh, int lsh, const HcPlan &h,
                                                   double *__restrict__ wsm, const S2klOut &so,
                                                   double *__restrict__ qsum, int lane)
{
    // grouped accumulation when the groups fit the lane's registers
    const int ng = (h.ngrp + 31) / 32;
    if (ng <= kHcMaxG) {
        if (h.ze == 1)
            eri_quartet_hcg<D, MODE, 32, 1>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, wsm, so, qsum, lane,
                                            kHcSmem, ng);
        else if (h.ze == 2)
            eri_quartet_hcg<D, MODE, 32, 2>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, wsm, so, qsum, lane,
                                            kHcSmem, ng);
        else
            eri_quartet_hcg<D, MODE, 32, 3>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, wsm, so, qsum, lane,
                                            kHcSmem, ng);
        return;
    }
    const int nj = (h.nacc + 31) / 32;
    if (nj <= 8)
        eri_quartet_hc<D, MODE, 8, 32>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, wsm, so, qsum, lane, kHcSmem);
    else if (nj <= 16)
        eri_quartet_hc<D, MODE, 16, 32>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, wsm, so, qsum, lane, kHcSmem);
    else if (nj <= 24)
        eri_quartet_hc<D, MODE, 24, 32>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, wsm, so, qsum, lane, kHcSmem);
    else if (nj <= 32)
        eri_quartet_hc<D, MODE, 32, 32>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, wsm, so, qsum, lane, kHcSmem);
    else
        eri_quartet_hc<D, MODE, kHcMaxJ, 32>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, wsm, so, qsum, lane,
                                             kHcSmem);
}

// Heavy quartets (CTA of 256 threads): up to 16 accumulators per thread.
static constexpr int kHcCtaMaxJ = 16;

template <int D, int MODE>
__device__ __forceinline__ void eri_quartet_hc_cta(const int *__restrict__ atm, const int *__restrict__ bas,
                                                   const double *__restrict__ env, const int *__restrict__ ao_loc,
                                                   int ish, int jsh, int ksh, int lsh, const HcPlan &h,
                                                   double *__restrict__ sm, int cap, const S2klOut &so,
                                                   double *__restrict__ qsum)
{
    const int ng = (h.ngrp + 255) / 256;
    if (ng <= 4) {
        if (h.ze == 1)
            eri_quartet_hcg<D, MODE, 256, 1>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, sm, so, qsum,
                                             threadIdx.x, cap, ng);
        else if (h.ze == 2)
            eri_quartet_hcg<D, MODE, 256, 2>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, sm, so, qsum,
                                             threadIdx.x, cap, ng);
        else
            eri_quartet_hcg<D, MODE, 256, 3>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, sm, so, qsum,
                                             threadIdx.x, cap, ng);
        return;
    }
    if (h.nacc <= 256 * 8)
        eri_quartet_hc<D, MODE, 8, 256>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, sm, so, qsum, threadIdx.x, cap);
    else
        eri_quartet_hc<D, MODE, kHcCtaMaxJ, 256>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, sm, so, qsum,
                                                 threadIdx.x, cap);
}

// Quartets whose Cartesian block has more functions than heavy_nf(D) go to
// the CTA-cooperative kernel; smaller ones are one warp each.  Measured on the
// 2^18-quartet benchmark set: int2e is fastest with the (dd|dp)-class blocks
// (648 functions) on warps, int2e_ip1 with them on CTAs (119 -> 89 ms).

__device__ __forceinline__ int quartet_nf(const int *__restrict__ bas, int i, int j, int k, int l)
{
    return ncart(bas[i * CB_BAS_SLOTS + CB_ANG_OF]) * ncart(bas[j * CB_BAS_SLOTS + CB_ANG_OF]) *
           ncart(bas[k * CB_BAS_SLOTS + CB_ANG_OF]) * ncart(bas[l * CB_BAS_SLOTS + CB_ANG_OF]);
}

// One heavy shell quartet per CTA (256 threads).  Same three phases as the
// warp kernel, with the CTA's threads sharing one slot batch (up to 64 slots)
// and the (output, component) entries spread 16 per thread in registers, so
// blocks of up to 4096 entries never recompute the recurrences; larger (l > 2)
// blocks are done in chunks of 4096 entries.
static constexpr int kHeavyAcc = 16;

template <int D, int MODE, bool LOW>
__device__ void eri_quartet_cta(const int *__restrict__ atm, const int *__restrict__ bas,
                                const double *__restrict__ env, const int *__restrict__ ao_loc, int ish, int jsh,
                                int ksh, int lsh, double *__restrict__ sm, int smem_doubles, const S2klOut &so,
                                double *__restrict__ qsum)
{
    constexpr int NC = D ? 3 : 1;
    const int tid = threadIdx.x;
    const Shell si = load_shell(atm, bas, env, ish), sj_ = load_shell(atm, bas, env, jsh);
    const Shell sk_ = load_shell(atm, bas, env, ksh), sl_ = load_shell(atm, bas, env, lsh);
    const int li = si.l, lj = sj_.l, lk = sk_.l, ll = sl_.l;
    const int nfi = ncart(li), nfj = ncart(lj), nfk = ncart(lk), nfl = ncart(ll);
    const int nf = nfi * nfj * nfk * nfl;
    const int ne = nf * NC;
    const int nroots = (li + lj + lk + ll + D) / 2 + 1;
    const int sj = li + 1 + D, sk = sj * (lj + 1), sl = sk * (lk + 1), gsz = sl * (ll + 1);
    double AB[3], CD[3];
    for (int x = 0; x < 3; x++) {
        AB[x] = si.R[x] - sj_.R[x];
        CD[x] = sk_.R[x] - sl_.R[x];
    }
    const double rab2 = AB[0] * AB[0] + AB[1] * AB[1] + AB[2] * AB[2];
    const double rcd2 = CD[0] * CD[0] + CD[1] * CD[1] + CD[2] * CD[2];
    const PairMask mb = pair_mask(si, sj_, rab2, li + lj + D), mk = pair_mask(sk_, sl_, rcd2, lk + ll);
    const int nslot = mb.n * mk.n * nroots;
    const double pref0 = 34.986836655249725693 * common_fac(li) * common_fac(lj) * common_fac(lk) * common_fac(ll);
    // shared memory: [pair rows][slot parameters][2D tables]
    const int gst = gsz | 1;     // odd per-direction table stride (bank spread)
    int tabn = (mb.n + mk.n) * kPairStride;
    if (tabn > smem_doubles / 4 || smem_doubles - tabn < 3 * gst + kParStride) tabn = 0;
    int ns = (smem_doubles - tabn) / (3 * gst + kParStride);
    ns = ns > kMaxSlots ? kMaxSlots : ns;
    double *tab = tabn ? sm : nullptr;
    double *par = sm + tabn;
    double *gbuf = par + ns * kParStride;
    if (tab) build_pair_tables(si, sj_, sk_, sl_, mb, mk, AB, rab2, CD, rcd2, tab, tid, kHeavyThreads);
    double qv[6] = {0, 0, 0, 0, 0, 0};

    for (int e0 = 0; e0 < ne; e0 += kHeavyThreads * kHeavyAcc) {
        double acc[kHeavyAcc];
        int gidx[kHeavyAcc];      // ax | ay << 10 | az << 20
        int ginfo[kHeavyAcc];     // component | ix << 2 | iy << 6 | iz << 10
#pragma unroll
        for (int n = 0; n < kHeavyAcc; n++) {
            acc[n] = 0.0;
            gidx[n] = 0;
            ginfo[n] = 0;
            const int e = e0 + tid + n * kHeavyThreads;
            if (e < ne) {
                const int f = e / NC, c = e - f * NC;
                int t = f;
                const int fl = t % nfl; t /= nfl;
                const int fk = t % nfk; t /= nfk;
                const int fj = t % nfj;
                const int fi = t / nfj;
                const int ci = c_cart[c_cart_off[li] + fi], cj = c_cart[c_cart_off[lj] + fj];
                const int ck = c_cart[c_cart_off[lk] + fk], cl = c_cart[c_cart_off[ll] + fl];
                const int ax = (ci & 15) + (cj & 15) * sj + (ck & 15) * sk + (cl & 15) * sl;
                const int ay = ((ci >> 4) & 15) + ((cj >> 4) & 15) * sj + ((ck >> 4) & 15) * sk + ((cl >> 4) & 15) * sl;
                const int az = (ci >> 8) + (cj >> 8) * sj + (ck >> 8) * sk + (cl >> 8) * sl;
                gidx[n] = ax | (ay << 10) | (az << 20);
                ginfo[n] = c | ((ci & 15) << 2) | (((ci >> 4) & 15) << 6) | ((ci >> 8) << 10);
            }
        }
        for (int s0 = 0; s0 < nslot; s0 += ns) {
            const int s1 = min(nslot, s0 + ns);
            __syncthreads();
            slot_params(tab, si, sj_, sk_, sl_, mb, mk, AB, rab2, CD, rcd2, nroots, pref0, s0, s1, par, tid,
                        kHeavyThreads);
            __syncthreads();
            for (int it = tid; it < (s1 - s0) * 3; it += kHeavyThreads) {
                const int s = it / 3, dir = it - s * 3;
                build_g_any<D, LOW>(par + s * kParStride, dir, li, lj, lk, ll, AB[dir], CD[dir],
                                    gbuf + (s * 3 + dir) * gst);
            }
            __syncthreads();
            for (int s = 0; s < s1 - s0; s++) {
                const double *gx = gbuf + s * 3 * gst, *gy = gx + gst, *gz = gy + gst;
                const double ai2 = par[s * kParStride + 10];
#pragma unroll
                for (int n = 0; n < kHeavyAcc; n++) {
                    if (e0 + tid + n * kHeavyThreads < ne) {
                        const int ax = gidx[n] & 1023, ay = (gidx[n] >> 10) & 1023, az = gidx[n] >> 20;
                        if (D == 0) {
                            acc[n] = fma(gx[ax] * gy[ay], gz[az], acc[n]);
                        } else {
                            const int c = ginfo[n] & 3;
                            const int ie = c == 0 ? (ginfo[n] >> 2) & 15 : (c == 1 ? (ginfo[n] >> 6) & 15 : ginfo[n] >> 10);
                            const double *gd = c == 0 ? gx : (c == 1 ? gy : gz);
                            const int ad = c == 0 ? ax : (c == 1 ? ay : az);
                            double fd = -ai2 * gd[ad + 1];
                            if (ie) fd = fma((double)ie, gd[ad - 1], fd);
                            const double px = c == 0 ? fd : gx[ax];
                            const double py = c == 1 ? fd : gy[ay];
                            const double pz = c == 2 ? fd : gz[az];
                            acc[n] = fma(px * py, pz, acc[n]);
                        }
                    }
                }
            }
        }
        // ---- epilogue of this chunk
        if (MODE == MODE_S2KL) {
            const int i0 = ao_loc[ish] - so.i_base, j0 = ao_loc[jsh], k0 = ao_loc[ksh], l0 = ao_loc[lsh];
#pragma unroll
            for (int n = 0; n < kHeavyAcc; n++) {
                const int e = e0 + tid + n * kHeavyThreads;
                if (e < ne) {
                    const int f = e / NC, c = e - f * NC;
                    int t = f;
                    const int fl = t % nfl; t /= nfl;
                    const int fk = t % nfk; t /= nfk;
                    const int fj = t % nfj;
                    const int fi = t / nfj;
                    if (ksh == lsh && fl > fk) continue;
                    const long long k = k0 + fk, l = l0 + fl;
                    so.out[c * so.comp_stride + ((long long)(i0 + fi) * so.nao + (j0 + fj)) * so.nao_pair +
                           k * (k + 1) / 2 + l] = acc[n];
                }
            }
        } else if (MODE == MODE_FULL) {
            const int i0 = ao_loc[ish], j0 = ao_loc[jsh], k0 = ao_loc[ksh], l0 = ao_loc[lsh];
#pragma unroll
            for (int n = 0; n < kHeavyAcc; n++) {
                const int e = e0 + tid + n * kHeavyThreads;
                if (e < ne) {
                    int t = e / NC;
                    const int fl = t % nfl; t /= nfl;
                    const int fk = t % nfk; t /= nfk;
                    const int fj = t % nfj;
                    const int fi = t / nfj;
                    full_store8(so.out, so.nao, i0 + fi, j0 + fj, k0 + fk, l0 + fl, acc[n]);
                }
            }
        } else if (MODE == MODE_GRAD) {
            const long long nao = so.nao;
            const int i0 = ao_loc[ish], j0 = ao_loc[jsh], k0 = ao_loc[ksh], l0 = ao_loc[lsh];
#pragma unroll
            for (int n = 0; n < kHeavyAcc; n++) {
                const int e = e0 + tid + n * kHeavyThreads;
                if (e < ne) {
                    const int f = e / NC, c = e - f * NC;
                    int t = f;
                    const int fl = t % nfl; t /= nfl;
                    const int fk = t % nfk; t /= nfk;
                    const int fj = t % nfj;
                    const int fi = t / nfj;
                    qv[c] = fma(acc[n], so.gamma_at(i0 + fi, j0 + fj, k0 + fk, l0 + fl), qv[c]);
                }
            }
        } else {
#pragma unroll
            for (int n = 0; n < kHeavyAcc; n++) {
                const int e = e0 + tid + n * kHeavyThreads;
                if (e < ne) {
                    const int f = e / NC, c = e - f * NC;
                    qv[2 * c] += acc[n] * (1.0 + 0.125 * (f & 7));
                    qv[2 * c + 1] += acc[n] * acc[n];
                }
            }
        }
    }
    if (MODE == MODE_QSUM || MODE == MODE_GRAD) {
        constexpr int NOUT = MODE == MODE_QSUM ? 2 * NC : NC;
        const double wkl = MODE == MODE_GRAD && ksh != lsh ? 2.0 : 1.0;
        __shared__ double red[kHeavyThreads / 32][6];
        for (int c = 0; c < NOUT; c++)
            for (int o = 16; o > 0; o >>= 1) qv[c] += __shfl_xor_sync(0xffffffffu, qv[c], o);
        __syncthreads();
        if ((tid & 31) == 0)
            for (int c = 0; c < NOUT; c++) red[tid >> 5][c] = qv[c];
        __syncthreads();
        if (tid == 0)
            for (int c = 0; c < NOUT; c++) {
                double t = 0.0;
                for (int w = 0; w < kHeavyThreads / 32; w++) t += red[w][c];
                qsum[c] = wkl * t;
            }
    }
}


// A quartet that an l <= 2 heavy kernel cannot place on the contracted-HRR
// path (none of the l <= 2 classes at the compiled shared-memory sizes; the
// per-output CTA path is left out of those kernels to save registers): its
// outputs are written as NaN so the failure cannot pass silently.
template <int D, int MODE>
__device__ void quartet_mark_bad(const int *__restrict__ bas, const int *__restrict__ ao_loc, int ish, int jsh,
                                 int ksh, int lsh, const S2klOut &so, double *__restrict__ qsum)
{
    constexpr int NC = D ? 3 : 1;
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    if (MODE == MODE_QSUM || MODE == MODE_GRAD) {
        if (threadIdx.x < (MODE == MODE_QSUM ? 2 * NC : NC)) qsum[threadIdx.x] = nan;
        return;
    }
    const int ni = ncart(bas[ish * CB_BAS_SLOTS + CB_ANG_OF]), nj = ncart(bas[jsh * CB_BAS_SLOTS + CB_ANG_OF]);
    const int nk = ncart(bas[ksh * CB_BAS_SLOTS + CB_ANG_OF]), nl = ncart(bas[lsh * CB_BAS_SLOTS + CB_ANG_OF]);
    for (int e = threadIdx.x; e < ni * nj * nk * nl; e += blockDim.x) {
        int t = e;
        const int fl = t % nl; t /= nl;
        const int fk = t % nk; t /= nk;
        const int fj = t % nj;
        const int fi = t / nj;
        if (MODE == MODE_FULL) {
            full_store8(so.out, so.nao, ao_loc[ish] + fi, ao_loc[jsh] + fj, ao_loc[ksh] + fk, ao_loc[lsh] + fl, nan);
        } else if (MODE == MODE_S2KL) {
            if (ksh == lsh && fl > fk) continue;
            const long long k = ao_loc[ksh] + fk, l = ao_loc[lsh] + fl;
            for (int c = 0; c < NC; c++)
                so.out[c * so.comp_stride + ((long long)(ao_loc[ish] - so.i_base + fi) * so.nao + (ao_loc[jsh] + fj)) *
                                                so.nao_pair + k * (k + 1) / 2 + l] = nan;
        }
    }
}

// s2kl block of shells [ish0, ish1) x all j x all k >= l (decontracted shells).
template <int D, bool LOW, bool SPH = false>
__global__ void __launch_bounds__(kWarps * 32, kWarpCtas) eri_s2kl_kernel(
    const int *__restrict__ atm, const int *__restrict__ bas, const double *__restrict__ env,
    const int *__restrict__ ao_loc, int ish0, int ish1, int nbas, int nao, double *__restrict__ out,
    int smem_warp, PathTable paths, const int *__restrict__ ao_sph = nullptr, const double *__restrict__ c2s = nullptr)
{
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *wsm = smem + warp * smem_warp;
    const long long npairs = (long long)nbas * (nbas + 1) / 2;
    const long long nq = (long long)(ish1 - ish0) * nbas * npairs;
    // SPH (l <= 2 kernels): spherical output, nao spherical AOs
    constexpr int M = SPH ? MODE_S2KL_SPH : MODE_S2KL;
    const int *oloc = SPH ? ao_sph : ao_loc;
    S2klOut so = {};
    so.out = out;
    so.nao = nao;
    so.nao_pair = (long long)nao * (nao + 1) / 2;
    so.comp_stride = (long long)(oloc[ish1] - oloc[ish0]) * nao * so.nao_pair;
    so.i_base = oloc[ish0];
    so.c2s = SPH ? c2s : nullptr;
    so.ao_sph = ao_sph;
    for (long long q = (long long)blockIdx.x * kWarps + warp; q < nq; q += (long long)gridDim.x * kWarps) {
        const long long ij = q / npairs;
        int ksh, lsh;
        decode_pair(q - ij * npairs, ksh, lsh);
        const int ish = ish0 + (int)(ij / nbas), jsh = (int)(ij % nbas);
        const int nfq = quartet_nf(bas, ish, jsh, ksh, lsh);
        if (nfq > heavy_nf(D)) continue;
        if (LOW) {
            HcPlan h;
            const int li = bas[ish * CB_BAS_SLOTS + CB_ANG_OF], lj = bas[jsh * CB_BAS_SLOTS + CB_ANG_OF];
            const int lk = bas[ksh * CB_BAS_SLOTS + CB_ANG_OF], ll = bas[lsh * CB_BAS_SLOTS + CB_ANG_OF];
            // spherical output stages the whole block: the per-output path
            // holds at most 256 functions, larger blocks take this path
            const int force = SPH && nfq > 256 ? 1 : paths.force(li, lj, lk, ll);
            if (hc_plan(D, li, lj, lk, ll, h, 32 * kHcMaxJ, kHcSmem, false, force)) {
                eri_quartet_hc_any<D, M>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, h, wsm, so, nullptr, lane);
                continue;
            }
        }
        eri_quartet_any<D, M, LOW>(atm, bas, env, ao_loc, ish, jsh, ksh, lsh, wsm, smem_warp, so, nullptr, lane,
                                           nfq);
    }
}

// Explicit quartet list (int4 shells): MODE_QSUM writes two checksums per
// component per quartet, MODE_GRAD one gamma contraction per component.
// heavy: quartets with more Cartesian functions than this go to the CTA kernel
// (0: heavy_nf(D)); the CTA kernel of the same list gets the same value.
template <int D, bool LOW, int MODE = MODE_QSUM>
__global__ void __launch_bounds__(warps_of(MODE) * 32, kWarpCtas * kWarps / warps_of(MODE)) eri_qsum_kernel(
    const int *__restrict__ atm, const int *__restrict__ bas, const double *__restrict__ env,
    const int4 *__restrict__ quartets, long long nq, double *__restrict__ qsum, int smem_warp,
    const int *__restrict__ ao_loc = nullptr, const double *__restrict__ gamma = nullptr, int nao = 0,
    double *__restrict__ full = nullptr, int heavy = 0, int grow0 = 0, int grows = 0, PathTable paths = {})
{
    if (heavy <= 0) heavy = heavy_nf(D);
    extern __shared__ double smem[];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double *wsm = smem + warp * smem_warp;
    S2klOut so = {};
    so.gamma = gamma;
    so.g_row0 = grow0;
    so.g_rows = grows > 0 ? grows : nao;
    so.out = full;                 // MODE_FULL output
    so.nao = nao;
    constexpr int NC = D ? 3 : 1;
    constexpr int NOUT = MODE == MODE_QSUM ? 2 * NC : NC;
    // lists are L-class ordered, cheap classes first: walk them from the end
    // so the expensive quartets start first and cheap ones fill the tail.  A
    // block takes one contiguous chunk, so its warps run the same class (and
    // code path) at the same time; inside the chunk each warp takes the next
    // quartet from a shared counter, so a warp that drew costly quartets
    // (many primitives) does not hold the block while the others idle.
    const long long per = (nq + gridDim.x - 1) / gridDim.x;
    const long long t0 = (long long)blockIdx.x * per, t1 = t0 + per < nq ? t0 + per : nq;
    __shared__ int next_q;
    if (threadIdx.x == 0) next_q = 0;
    __syncthreads();
    for (;;) {
        int k = 0;
        if (lane == 0) k = atomicAdd(&next_q, 1);
        k = __shfl_sync(0xffffffffu, k, 0);
        const long long t = t0 + k;
        if (t >= t1) break;
        const long long q = nq - 1 - t;
        const int4 s = quartets[q];
        const int nfq = quartet_nf(bas, s.x, s.y, s.z, s.w);
        if (nfq > heavy) continue;
        double acc[NOUT];
        for (int c = 0; c < NOUT; c++) acc[c] = 0.0;
        HcPlan h;
        const int li = bas[s.x * CB_BAS_SLOTS + CB_ANG_OF], lj = bas[s.y * CB_BAS_SLOTS + CB_ANG_OF];
        const int lk = bas[s.z * CB_BAS_SLOTS + CB_ANG_OF], ll = bas[s.w * CB_BAS_SLOTS + CB_ANG_OF];
        if (LOW && hc_plan(D, li, lj, lk, ll, h, 32 * kHcMaxJ, kHcSmem, false, paths.force(li, lj, lk, ll)))
            eri_quartet_hc_any<D, MODE>(atm, bas, env, ao_loc, s.x, s.y, s.z, s.w, h, wsm, so, acc, lane);
        else
            eri_quartet_any<D, MODE, LOW>(atm, bas, env, ao_loc, s.x, s.y, s.z, s.w, wsm, smem_warp, so, acc, lane,
                                          nfq);
        if (lane == 0)
            for (int c = 0; c < NOUT; c++)
                if (MODE != MODE_FULL) qsum[q * NOUT + c] = acc[c];
    }
}

// Heavy quartets of the s2kl block (explicit list built by the caller).
template <int D, bool LOW, bool SPH = false>
__global__ void __launch_bounds__(kHeavyThreads, 1) eri_s2kl_heavy_kernel(
    const int *__restrict__ atm, const int *__restrict__ bas, const double *__restrict__ env,
    const int *__restrict__ ao_loc, int ish0, int ish1, int nao, const int4 *__restrict__ quartets, long long nq,
    double *__restrict__ out, int smem_doubles, const int *__restrict__ ao_sph = nullptr,
    const double *__restrict__ c2s = nullptr)
{
    extern __shared__ double smem[];
    constexpr int M = SPH ? MODE_S2KL_SPH : MODE_S2KL;
    const int *oloc = SPH ? ao_sph : ao_loc;
    S2klOut so = {};
    so.out = out;
    so.nao = nao;
    so.nao_pair = (long long)nao * (nao + 1) / 2;
    so.comp_stride = (long long)(oloc[ish1] - oloc[ish0]) * nao * so.nao_pair;
    so.i_base = oloc[ish0];
    so.c2s = SPH ? c2s : nullptr;
    so.ao_sph = ao_sph;
    for (long long q = blockIdx.x; q < nq; q += gridDim.x) {
        const int4 s = quartets[q];
        HcPlan h;
        const int li = bas[s.x * CB_BAS_SLOTS + CB_ANG_OF], lj = bas[s.y * CB_BAS_SLOTS + CB_ANG_OF];
        const int lk = bas[s.z * CB_BAS_SLOTS + CB_ANG_OF], ll = bas[s.w * CB_BAS_SLOTS + CB_ANG_OF];
        if (LOW && hc_plan(D, li, lj, lk, ll, h, 256 * kHcCtaMaxJ, smem_doubles, true)) {
            eri_quartet_hc_cta<D, M>(atm, bas, env, ao_loc, s.x, s.y, s.z, s.w, h, smem, smem_doubles, so,
                                             nullptr);
            continue;
        }
        if (SPH) {   // spherical output needs the contracted-HRR path: mark the block
            s2kl_sph_store<kHeavyThreads>(smem, smem, D ? 3 : 1, li, lj, lk, ll, s.x, s.y, s.z, s.w, so, threadIdx.x,
                                          true);
            continue;
        }
        if constexpr (LOW)
            quartet_mark_bad<D, MODE_S2KL>(bas, ao_loc, s.x, s.y, s.z, s.w, so, nullptr);
        else
            eri_quartet_cta<D, MODE_S2KL, LOW>(atm, bas, env, ao_loc, s.x, s.y, s.z, s.w, smem, smem_doubles, so,
                                               nullptr);
    }
}

// Heavy quartets of an explicit list (light ones are skipped here).
template <int D, bool LOW, int MODE = MODE_QSUM>
__global__ void __launch_bounds__(kHeavyThreads, 1) eri_qsum_heavy_kernel(
    const int *__restrict__ atm, const int *__restrict__ bas, const double *__restrict__ env,
    const int4 *__restrict__ quartets, long long nq, double *__restrict__ qsum, int smem_doubles,
    const int *__restrict__ ao_loc = nullptr, const double *__restrict__ gamma = nullptr, int nao = 0,
    double *__restrict__ full = nullptr, int heavy = 0, int grow0 = 0, int grows = 0)
{
    if (heavy <= 0) heavy = heavy_nf(D);
    extern __shared__ double smem[];
    S2klOut so = {};
    so.gamma = gamma;
    so.g_row0 = grow0;
    so.g_rows = grows > 0 ? grows : nao;
    so.out = full;                 // MODE_FULL output
    so.nao = nao;
    constexpr int NC = D ? 3 : 1;
    constexpr int NOUT = MODE == MODE_QSUM ? 2 * NC : NC;
    // The CTA's quartets are q = blockIdx.x + k gridDim.x.  They are screened
    // for heavy ones kHeavyThreads at a time, one per thread, and compacted in
    // shared memory (list order kept), so finding the heavy quartets costs one
    // parallel load per kHeavyThreads list entries instead of a serial chain of
    // dependent loads over every entry.
    __shared__ int hq[kHeavyThreads];
    __shared__ int wcnt[kHeavyThreads / 32];
    const int tid = threadIdx.x, hl = tid & 31, hw = tid >> 5;
    for (long long base = blockIdx.x; base < nq; base += (long long)gridDim.x * kHeavyThreads) {
        const long long qt = base + (long long)tid * gridDim.x;
        bool hv = false;
        if (qt < nq) {
            const int4 t = quartets[qt];
            hv = quartet_nf(bas, t.x, t.y, t.z, t.w) > heavy;
        }
        const unsigned m = __ballot_sync(0xffffffffu, hv);
        if (hl == 0) wcnt[hw] = __popc(m);
        __syncthreads();
        int off = 0, nh = 0;
        for (int w = 0; w < kHeavyThreads / 32; w++) {
            if (w < hw) off += wcnt[w];
            nh += wcnt[w];
        }
        if (hv) hq[off + __popc(m & ((1u << hl) - 1u))] = tid;
        __syncthreads();
        for (int ih = 0; ih < nh; ih++) {
            const long long q = base + (long long)hq[ih] * gridDim.x;
            const int4 s = quartets[q];
            HcPlan h;
            if (LOW && hc_plan(D, bas[s.x * CB_BAS_SLOTS + CB_ANG_OF], bas[s.y * CB_BAS_SLOTS + CB_ANG_OF],
                               bas[s.z * CB_BAS_SLOTS + CB_ANG_OF], bas[s.w * CB_BAS_SLOTS + CB_ANG_OF], h,
                               256 * kHcCtaMaxJ, smem_doubles, true)) {
                eri_quartet_hc_cta<D, MODE>(atm, bas, env, ao_loc, s.x, s.y, s.z, s.w, h, smem, smem_doubles, so,
                                            MODE == MODE_FULL ? nullptr : qsum + q * NOUT);
                continue;
            }
            if constexpr (LOW)
                quartet_mark_bad<D, MODE>(bas, ao_loc, s.x, s.y, s.z, s.w, so,
                                          MODE == MODE_FULL ? nullptr : qsum + q * NOUT);
            else
                eri_quartet_cta<D, MODE, LOW>(atm, bas, env, ao_loc, s.x, s.y, s.z, s.w, smem, smem_doubles, so,
                                              MODE == MODE_FULL ? nullptr : qsum + q * NOUT);
        }
        __syncthreads();    // hq, wcnt are rewritten by the next screening step
    }
}

template <typename K>
static inline int prepare_kernel(K kernel, size_t smem)
{
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) {
            set_error("cudaFuncSetAttribute: %s", cudaGetErrorString(e));
            return CCSD_B200_ERR_LAUNCH;
        }
    }
    return CCSD_B200_OK;
}


// ---- launchers (instantiated per (D, LOW) in eri_inst_*.cu) ----
template <int D, bool LOW>
int launch_s2kl(const EriArgs &a, long long grid, size_t smem, cudaStream_t st)
{
    int rc;
    if constexpr (LOW) {
        if (a.c2s) {
            if ((rc = prepare_kernel(eri_s2kl_kernel<D, LOW, true>, smem))) return rc;
            eri_s2kl_kernel<D, LOW, true><<<(int)grid, kWarps * 32, smem, st>>>(
                a.atm, a.bas, a.env, a.ao_loc, a.ish0, a.ish1, a.nbas, a.nao, a.out, a.smem_warp, a.paths, a.ao_sph,
                a.c2s);
            return check_launch("eri_s2kl_kernel");
        }
    }
    if ((rc = prepare_kernel(eri_s2kl_kernel<D, LOW>, smem))) return rc;
    eri_s2kl_kernel<D, LOW><<<(int)grid, kWarps * 32, smem, st>>>(a.atm, a.bas, a.env, a.ao_loc, a.ish0, a.ish1,
                                                                  a.nbas, a.nao, a.out, a.smem_warp,
                                                                  a.paths, a.ao_sph, a.c2s);
    return check_launch("eri_s2kl_kernel");
}

template <int D, bool LOW>
int launch_s2kl_heavy(const EriArgs &a, long long grid, size_t smem, cudaStream_t st)
{
    int rc;
    if constexpr (LOW) {
        if (a.c2s) {
            if ((rc = prepare_kernel(eri_s2kl_heavy_kernel<D, LOW, true>, smem))) return rc;
            eri_s2kl_heavy_kernel<D, LOW, true><<<(int)grid, kHeavyThreads, smem, st>>>(
                a.atm, a.bas, a.env, a.ao_loc, a.ish0, a.ish1, a.nao, a.quartets, a.nq, a.out, a.smem_heavy, a.ao_sph,
                a.c2s);
            return check_launch("eri_s2kl_heavy_kernel");
        }
    }
    if ((rc = prepare_kernel(eri_s2kl_heavy_kernel<D, LOW>, smem))) return rc;
    eri_s2kl_heavy_kernel<D, LOW><<<(int)grid, kHeavyThreads, smem, st>>>(a.atm, a.bas, a.env, a.ao_loc, a.ish0,
                                                                          a.ish1, a.nao, a.quartets, a.nq, a.out,
                                                                          a.smem_heavy, a.ao_sph, a.c2s);
    return check_launch("eri_s2kl_heavy_kernel");
}

template <int D, bool LOW, int MODE>
int launch_list(const EriArgs &a, long long grid, size_t smem, cudaStream_t st)
{
    int rc;
    if ((rc = prepare_kernel(eri_qsum_kernel<D, LOW, MODE>, smem))) return rc;
    eri_qsum_kernel<D, LOW, MODE><<<(int)grid, warps_of(MODE) * 32, smem, st>>>(a.atm, a.bas, a.env, a.quartets, a.nq,
                                                                        a.qsum, a.smem_warp, a.ao_loc, a.gamma,
                                                                        a.nao, a.full, a.heavy, a.grow0, a.grows,
                                                                        a.paths);
    return check_launch("eri_qsum_kernel");
}

template <int D, bool LOW, int MODE>
int launch_list_heavy(const EriArgs &a, long long grid, size_t smem, cudaStream_t st)
{
    int rc;
    if ((rc = prepare_kernel(eri_qsum_heavy_kernel<D, LOW, MODE>, smem))) return rc;
    eri_qsum_heavy_kernel<D, LOW, MODE><<<(int)grid, kHeavyThreads, smem, st>>>(
        a.atm, a.bas, a.env, a.quartets, a.nq, a.qsum, a.smem_heavy, a.ao_loc, a.gamma, a.nao, a.full, a.heavy,
        a.grow0, a.grows);
    return check_launch("eri_qsum_heavy_kernel");
}

#define CB_ERI_INSTANTIATE(DV, LOWV)                                                                           \
    template int launch_s2kl<DV, LOWV>(const EriArgs &, long long, size_t, cudaStream_t);                      \
    template int launch_s2kl_heavy<DV, LOWV>(const EriArgs &, long long, size_t, cudaStream_t);                \
    template int launch_list<DV, LOWV, MODE_QSUM>(const EriArgs &, long long, size_t, cudaStream_t);           \
    template int launch_list_heavy<DV, LOWV, MODE_QSUM>(const EriArgs &, long long, size_t, cudaStream_t);     \
    template int launch_list<DV, LOWV, (DV ? MODE_GRAD : MODE_FULL)>(const EriArgs &, long long, size_t,        \
                                                                      cudaStream_t);                            \
    template int launch_list_heavy<DV, LOWV, (DV ? MODE_GRAD : MODE_FULL)>(const EriArgs &, long long, size_t,  \
                                                                            cudaStream_t);

}  // namespace cb
