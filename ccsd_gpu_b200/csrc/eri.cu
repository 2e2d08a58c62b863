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
#include "common.cuh"
#include "eri_launch.h"

#include <atomic>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

namespace cb {

static char g_err[512] = "";

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

int check_launch(const char *what)
{
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_error("%s: %s", what, cudaGetErrorString(e));
        return CCSD_B200_ERR_LAUNCH;
    }
    return CCSD_B200_OK;
}

// out[s][c] = sum over quartets q in [seg[s], seg[s+1]) of qv[q][c], c < 3,
// summed in a fixed order (one CTA per segment, fixed-shape tree).
__global__ void segment_sum3_kernel(const double *__restrict__ qv, const long long *__restrict__ seg,
                                    double *__restrict__ out)
{
    __shared__ double red[3][256];
    const int s = blockIdx.x, tid = threadIdx.x;
    double a[3] = {0.0, 0.0, 0.0};
    for (long long q = seg[s] + tid; q < seg[s + 1]; q += 256)
        for (int c = 0; c < 3; c++) a[c] += qv[q * 3 + c];
    for (int c = 0; c < 3; c++) red[c][tid] = a[c];
    __syncthreads();
    for (int h = 128; h > 0; h >>= 1) {
        if (tid < h)
            for (int c = 0; c < 3; c++) red[c][tid] += red[c][tid + h];
        __syncthreads();
    }
    if (tid < 3) out[s * 3 + tid] = red[tid][0];
}

// ---- Cartesian -> spherical transform of an s2kl block (two passes) ----
// Sparse block-diagonal cart2sph: spherical AO s has coefficients
// val[ptr[s]..ptr[s+1]) on Cartesian AOs idx[...].

// pass 1: (ncomp, nfc, naoc, npc) -> (ncomp, nfs, naos, npc), transforms i and j
__global__ void c2s_ij_kernel(const double *__restrict__ in, double *__restrict__ out, int ncomp,
                              int nfc, int naoc, long long npc, int nfs, int naos,
                              const int *__restrict__ ptr_i, const int *__restrict__ idx_i,
                              const double *__restrict__ val_i, const int *__restrict__ ptr,
                              const int *__restrict__ idx, const double *__restrict__ val)
{
    const long long total = (long long)ncomp * nfs * naos * npc;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long kl = e % npc;
        long long t = e / npc;
        const int js = (int)(t % naos);
        t /= naos;
        const int is = (int)(t % nfs);
        const int c = (int)(t / nfs);
        double acc = 0.0;
        for (int a = ptr_i[is]; a < ptr_i[is + 1]; a++)
            for (int b = ptr[js]; b < ptr[js + 1]; b++)
                acc += val_i[a] * val[b] * in[(((long long)c * nfc + idx_i[a]) * naoc + idx[b]) * npc + kl];
        out[e] = acc;
    }
}

// pass 2: (rows, npc) -> (rows, nps), transforms k and l with s2 symmetry
__global__ void c2s_kl_kernel(const double *__restrict__ in, double *__restrict__ out, long long rows,
                              long long npc, int naos, const int *__restrict__ ptr,
                              const int *__restrict__ idx, const double *__restrict__ val)
{
    const long long nps = (long long)naos * (naos + 1) / 2;
    const long long total = rows * nps;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total;
         e += (long long)gridDim.x * blockDim.x) {
        const long long r = e / nps, p = e - r * nps;
        int ks, ls;
        decode_pair(p, ks, ls);
        const double *row = in + r * npc;
        double acc = 0.0;
        for (int a = ptr[ks]; a < ptr[ks + 1]; a++)
            for (int b = ptr[ls]; b < ptr[ls + 1]; b++) {
                const long long kc = idx[a], lc = idx[b];
                const long long pc = kc >= lc ? kc * (kc + 1) / 2 + lc : lc * (lc + 1) / 2 + kc;
                acc += val[a] * val[b] * row[pc];
            }
        out[e] = acc;
    }
}

static int smem_per_warp(int lmax, int deriv)
{
    const int gsz = (lmax + 1 + deriv) * (lmax + 1) * (lmax + 1) * (lmax + 1);
    int need = 3 * (gsz | 1) + kParStride;
    if (lmax <= 2 && need < kHcSmem) need = kHcSmem;     // contracted-HRR path
    return need < 2048 ? 2048 : need;
}

// shared memory of the CTA kernel: up to 64 slots of the largest class, <= 200 KiB
static int heavy_smem_doubles(int lmax, int deriv)
{
    const int gsz = (lmax + 1 + deriv) * (lmax + 1) * (lmax + 1) * (lmax + 1);
    const long long want = (long long)(lmax <= 2 ? kMaxSlotsCta : kMaxSlots) * (3 * (gsz | 1) + kParStride);
    const long long cap = 200 * 1024 / 8;
    return (int)(want < cap ? want : cap);
}

// Library-owned auxiliary stream per device: the heavy-quartet kernel runs on
// it, fork/joined with the caller's stream by events, so it overlaps the warp
// kernel instead of serialising behind it.
struct AuxStream {
    cudaStream_t s = nullptr;
    cudaEvent_t fork = nullptr, join = nullptr;
};

static int aux_stream(AuxStream **out)
{
    static AuxStream aux[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        set_error("aux_stream: no current CUDA device");
        return CCSD_B200_ERR_LAUNCH;
    }
    AuxStream &a = aux[dev];
    if (!a.s) {
        if (cudaStreamCreateWithFlags(&a.s, cudaStreamNonBlocking) != cudaSuccess ||
            cudaEventCreateWithFlags(&a.fork, cudaEventDisableTiming) != cudaSuccess ||
            cudaEventCreateWithFlags(&a.join, cudaEventDisableTiming) != cudaSuccess) {
            set_error("aux_stream: stream/event creation failed");
            a.s = nullptr;
            return CCSD_B200_ERR_LAUNCH;
        }
    }
    *out = &a;
    return CCSD_B200_OK;
}

static int num_sms()
{
    static int n = 0;
    if (!n) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        if (n <= 0) n = 148;
    }
    return n;
}


enum class Kind { S2KL, QSUM, GRAD, FULL };

template <int D, bool LOW>
static int launch_pair_dl(Kind k, const EriArgs &a, long long grid, size_t smem, long long hgrid, size_t hsmem,
                          cudaStream_t st, cudaStream_t hst)
{
    int rc = CCSD_B200_OK;
    if (hgrid > 0) {
        switch (k) {
        case Kind::S2KL: rc = launch_s2kl_heavy<D, LOW>(a, hgrid, hsmem, hst); break;
        case Kind::QSUM: rc = launch_list_heavy<D, LOW, MODE_QSUM>(a, hgrid, hsmem, hst); break;
        case Kind::GRAD: rc = D ? launch_list_heavy<D, LOW, MODE_GRAD>(a, hgrid, hsmem, hst) : CCSD_B200_ERR_ARG; break;
        case Kind::FULL: rc = D ? CCSD_B200_ERR_ARG : launch_list_heavy<D, LOW, MODE_FULL>(a, hgrid, hsmem, hst); break;
        }
        if (rc) return rc;
    }
    return CCSD_B200_OK;
}

template <int D, bool LOW>
static int launch_main_dl(Kind k, const EriArgs &a, long long grid, size_t smem, cudaStream_t st)
{
    switch (k) {
    case Kind::S2KL: return launch_s2kl<D, LOW>(a, grid, smem, st);
    case Kind::QSUM: return launch_list<D, LOW, MODE_QSUM>(a, grid, smem, st);
    case Kind::GRAD: return D ? launch_list<D, LOW, MODE_GRAD>(a, grid, smem, st) : CCSD_B200_ERR_ARG;
    case Kind::FULL: return D ? CCSD_B200_ERR_ARG : launch_list<D, LOW, MODE_FULL>(a, grid, smem, st);
    }
    return CCSD_B200_ERR_ARG;
}

// Accumulation path per L-class of the warp kernels, per derivative order
// (all zero: the measured rule); set by the autotuner.
static PathTable g_paths[2];

// The warp kernel over `nwork` quartets on the caller's stream and, when
// `nheavy` > 0, the CTA (heavy-quartet) kernel on the auxiliary stream,
// fork/joined by events so the two overlap.
static int run_pair(Kind k, int deriv, bool low, const EriArgs &a_in, long long nwork, long long nheavy,
                    cudaStream_t st)
{
    EriArgs a = a_in;
    a.paths = g_paths[deriv ? 1 : 0];
    const int nw = warps_of(k == Kind::GRAD ? MODE_GRAD : (k == Kind::FULL ? MODE_FULL : MODE_QSUM));
    const size_t smem = (size_t)a.smem_warp * nw * sizeof(double);
    long long grid = (nwork + nw - 1) / nw;
    const long long gmax = (long long)num_sms() * 16;
    if (grid > gmax) grid = gmax;
    const size_t hsmem = (size_t)a.smem_heavy * sizeof(double);
    const long long hg = nheavy < (long long)num_sms() ? nheavy : (long long)num_sms();
    int rc;
    AuxStream *aux = nullptr;
    if (nheavy > 0) {
        if ((rc = aux_stream(&aux))) return rc;
        cudaEventRecord(aux->fork, st);
        cudaStreamWaitEvent(aux->s, aux->fork, 0);
        if (deriv)
            rc = low ? launch_pair_dl<1, true>(k, a, grid, smem, hg, hsmem, st, aux->s)
                     : launch_pair_dl<1, false>(k, a, grid, smem, hg, hsmem, st, aux->s);
        else
            rc = low ? launch_pair_dl<0, true>(k, a, grid, smem, hg, hsmem, st, aux->s)
                     : launch_pair_dl<0, false>(k, a, grid, smem, hg, hsmem, st, aux->s);
        if (rc) return rc;
        cudaEventRecord(aux->join, aux->s);
    }
    if (deriv)
        rc = low ? launch_main_dl<1, true>(k, a, grid, smem, st) : launch_main_dl<1, false>(k, a, grid, smem, st);
    else
        rc = low ? launch_main_dl<0, true>(k, a, grid, smem, st) : launch_main_dl<0, false>(k, a, grid, smem, st);
    if (aux) cudaStreamWaitEvent(st, aux->join, 0);
    return rc;
}
}  // namespace cb

using namespace cb;

extern "C" {

const char *ccsd_b200_last_error(void) { return g_err; }

int ccsd_b200_eri_s2kl_cart(int deriv, const int32_t *atm, const int32_t *bas, const double *env, int nbas,
                            const int32_t *ao_loc, int ish0, int ish1, int nao, int lmax,
                            const int32_t *heavy_quartets, long long n_heavy, double *out, void *stream)
{
    if (deriv < 0 || deriv > 1 || !atm || !bas || !env || !ao_loc || !out || nbas <= 0 || ish0 < 0 ||
        ish1 > nbas || ish0 >= ish1 || nao <= 0 || lmax < 0 || n_heavy < 0 || (n_heavy > 0 && !heavy_quartets)) {
        set_error("ccsd_b200_eri_s2kl_cart: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    if (lmax > CB_LMAX) {
        set_error("ccsd_b200_eri_s2kl_cart: l = %d > %d is not supported", lmax, CB_LMAX);
        return CCSD_B200_ERR_UNSUPPORTED;
    }
    EriArgs a;
    a.atm = atm;
    a.bas = bas;
    a.env = env;
    a.ao_loc = ao_loc;
    a.ish0 = ish0;
    a.ish1 = ish1;
    a.nbas = nbas;
    a.nao = nao;
    a.out = out;
    a.quartets = reinterpret_cast<const int4 *>(heavy_quartets);
    a.nq = n_heavy;
    a.smem_warp = smem_per_warp(lmax, deriv);
    a.smem_heavy = heavy_smem_doubles(lmax, deriv);
    const long long nq = (long long)(ish1 - ish0) * nbas * ((long long)nbas * (nbas + 1) / 2);
    return run_pair(Kind::S2KL, deriv, lmax <= 2, a, nq, n_heavy, (cudaStream_t)stream);
}

int ccsd_b200_eri_s2kl_sph(int deriv, const int32_t *atm, const int32_t *bas, const double *env, int nbas,
                           const int32_t *ao_loc, const int32_t *ao_loc_sph, const double *c2s_d, int ish0, int ish1,
                           int nao_sph, int lmax, const int32_t *heavy_quartets, long long n_heavy, double *out,
                           void *stream)
{
    if (deriv < 0 || deriv > 1 || !atm || !bas || !env || !ao_loc || !ao_loc_sph || !c2s_d || !out || nbas <= 0 ||
        ish0 < 0 || ish1 > nbas || ish0 >= ish1 || nao_sph <= 0 || lmax < 0 || n_heavy < 0 ||
        (n_heavy > 0 && !heavy_quartets)) {
        set_error("ccsd_b200_eri_s2kl_sph: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    if (lmax > 2) {
        set_error("ccsd_b200_eri_s2kl_sph: l = %d > 2 (use ccsd_b200_eri_s2kl_cart + ccsd_b200_cart2sph_s2kl)",
                  lmax);
        return CCSD_B200_ERR_UNSUPPORTED;
    }
    EriArgs a;
    a.atm = atm;
    a.bas = bas;
    a.env = env;
    a.ao_loc = ao_loc;
    a.ish0 = ish0;
    a.ish1 = ish1;
    a.nbas = nbas;
    a.nao = nao_sph;
    a.out = out;
    a.quartets = reinterpret_cast<const int4 *>(heavy_quartets);
    a.nq = n_heavy;
    a.ao_sph = ao_loc_sph;
    a.c2s = c2s_d;
    a.smem_warp = smem_per_warp(lmax, deriv);
    a.smem_heavy = heavy_smem_doubles(lmax, deriv);
    const long long nq = (long long)(ish1 - ish0) * nbas * ((long long)nbas * (nbas + 1) / 2);
    return run_pair(Kind::S2KL, deriv, true, a, nq, n_heavy, (cudaStream_t)stream);
}

// Heavy-quartet thresholds of the list entry points (quartet checksums, the
// ip1 gradient contraction, the dense int2e tensor), per derivative order;
// set by the autotuner.  The s2kl block entry keeps the compiled values (its
// heavy list is built by the caller).
static int g_heavy_list[2] = {kHeavyNf, kHeavyNfIp1};

int ccsd_b200_eri_set_heavy_nf(int deriv, int nf)
{
    if (deriv < 0 || deriv > 1 || nf < 1) {
        set_error("ccsd_b200_eri_set_heavy_nf: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    g_heavy_list[deriv] = nf;
    return CCSD_B200_OK;
}

int ccsd_b200_eri_get_heavy_nf(int deriv)
{
    return deriv == 0 || deriv == 1 ? g_heavy_list[deriv] : -1;
}

int ccsd_b200_eri_set_paths(int deriv, const uint8_t *choice, int n)
{
    if (deriv < 0 || deriv > 1 || !choice || n != 81) {
        set_error("ccsd_b200_eri_set_paths: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    PathTable t;
    for (int c = 0; c < 81; c++) {
        if (choice[c] > 2) {
            set_error("ccsd_b200_eri_set_paths: choice[%d] = %d (0, 1 or 2)", c, (int)choice[c]);
            return CCSD_B200_ERR_ARG;
        }
        if (choice[c] == 1) t.hc[c >> 6] |= 1ull << (c & 63);
        if (choice[c] == 2) t.po[c >> 6] |= 1ull << (c & 63);
    }
    g_paths[deriv] = t;
    return CCSD_B200_OK;
}

int ccsd_b200_eri_get_paths(int deriv, uint8_t *choice, int n)
{
    if (deriv < 0 || deriv > 1 || !choice || n != 81) {
        set_error("ccsd_b200_eri_get_paths: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    for (int c = 0; c < 81; c++)
        choice[c] = (uint8_t)g_paths[deriv].force(c / 27, (c / 9) % 3, (c / 3) % 3, c % 3);
    return CCSD_B200_OK;
}

int ccsd_b200_eri_quartet_checksums(int deriv, const int32_t *atm, const int32_t *bas, const double *env,
                                    const int32_t *quartets, long long nq, int lmax, double *qsum,
                                    void *stream)
{
    if (deriv < 0 || deriv > 1 || !atm || !bas || !env || !quartets || !qsum || nq < 0 || lmax < 0) {
        set_error("ccsd_b200_eri_quartet_checksums: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    if (lmax > CB_LMAX) {
        set_error("ccsd_b200_eri_quartet_checksums: l = %d > %d is not supported", lmax, CB_LMAX);
        return CCSD_B200_ERR_UNSUPPORTED;
    }
    if (nq == 0) return CCSD_B200_OK;
    EriArgs a;
    a.atm = atm;
    a.bas = bas;
    a.env = env;
    a.quartets = reinterpret_cast<const int4 *>(quartets);
    a.nq = nq;
    a.qsum = qsum;
    a.heavy = g_heavy_list[deriv];
    a.smem_warp = smem_per_warp(lmax, deriv);
    a.smem_heavy = heavy_smem_doubles(lmax, deriv);
    return run_pair(Kind::QSUM, deriv, lmax <= 2, a, nq, nq, (cudaStream_t)stream);
}

int ccsd_b200_eri_ip1_contract_rows(const int32_t *atm, const int32_t *bas, const double *env,
                                    const int32_t *ao_loc, int nao, const double *gamma_rows, int row0, int nrows,
                                    const int32_t *quartets, long long nq, const long long *seg, int nseg, int lmax,
                                    double *qwork, double *out, void *stream)
{
    if (!atm || !bas || !env || !ao_loc || nao <= 0 || !gamma_rows || row0 < 0 || nrows <= 0 || row0 + nrows > nao ||
        !quartets || nq < 0 || !seg || nseg <= 0 || lmax < 0 || !qwork || !out) {
        set_error("ccsd_b200_eri_ip1_contract: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    if (lmax > CB_LMAX) {
        set_error("ccsd_b200_eri_ip1_contract: l = %d > %d is not supported", lmax, CB_LMAX);
        return CCSD_B200_ERR_UNSUPPORTED;
    }
    cudaStream_t st = (cudaStream_t)stream;
    int rc;
    if (nq > 0) {
        EriArgs a;
        a.atm = atm;
        a.bas = bas;
        a.env = env;
        a.ao_loc = ao_loc;
        a.nao = nao;
        a.gamma = gamma_rows;
        a.grow0 = row0;
        a.grows = nrows;
        a.quartets = reinterpret_cast<const int4 *>(quartets);
        a.nq = nq;
        a.qsum = qwork;
        a.heavy = g_heavy_list[1];
        a.smem_warp = smem_per_warp(lmax, 1);
        a.smem_heavy = heavy_smem_doubles(lmax, 1);
        if ((rc = run_pair(Kind::GRAD, 1, lmax <= 2, a, nq, nq, st))) return rc;
    }
    segment_sum3_kernel<<<nseg, 256, 0, st>>>(qwork, seg, out);
    return check_launch("segment_sum3_kernel");
}

int ccsd_b200_eri_ip1_contract(const int32_t *atm, const int32_t *bas, const double *env, const int32_t *ao_loc,
                               int nao, const double *gamma, const int32_t *quartets, long long nq,
                               const long long *seg, int nseg, int lmax, double *qwork, double *out, void *stream)
{
    return ccsd_b200_eri_ip1_contract_rows(atm, bas, env, ao_loc, nao, gamma, 0, nao, quartets, nq, seg, nseg, lmax,
                                           qwork, out, stream);
}

int ccsd_b200_eri_full_cart(const int32_t *atm, const int32_t *bas, const double *env, const int32_t *ao_loc,
                            int nao, const int32_t *quartets, long long nq, int lmax, double *out, void *stream)
{
    if (!atm || !bas || !env || !ao_loc || nao <= 0 || !quartets || nq < 0 || lmax < 0 || !out) {
        set_error("ccsd_b200_eri_full_cart: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    if (lmax > CB_LMAX) {
        set_error("ccsd_b200_eri_full_cart: l = %d > %d is not supported", lmax, CB_LMAX);
        return CCSD_B200_ERR_UNSUPPORTED;
    }
    if (nq == 0) return CCSD_B200_OK;
    EriArgs a;
    a.atm = atm;
    a.bas = bas;
    a.env = env;
    a.ao_loc = ao_loc;
    a.nao = nao;
    a.quartets = reinterpret_cast<const int4 *>(quartets);
    a.nq = nq;
    a.full = out;
    a.heavy = g_heavy_list[0];
    a.smem_warp = smem_per_warp(lmax, 0);
    a.smem_heavy = heavy_smem_doubles(lmax, 0);
    return run_pair(Kind::FULL, 0, lmax <= 2, a, nq, nq, (cudaStream_t)stream);
}

int ccsd_b200_cart2sph_s2kl(const double *cart, double *tmp, double *out, int ncomp, int nfc, int naoc, int nfs,
                            int naos, const int32_t *ptr_i, const int32_t *idx_i, const double *val_i,
                            const int32_t *ptr, const int32_t *idx, const double *val, void *stream)
{
    if (!cart || !tmp || !out || ncomp <= 0 || nfc <= 0 || naoc <= 0 || nfs <= 0 || naos <= 0 || !ptr_i ||
        !idx_i || !val_i || !ptr || !idx || !val) {
        set_error("ccsd_b200_cart2sph_s2kl: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    cudaStream_t st = (cudaStream_t)stream;
    const long long npc = (long long)naoc * (naoc + 1) / 2;
    const long long rows = (long long)ncomp * nfs * naos;
    const long long t1 = rows * npc;
    const int bs = 256;
    long long g1 = (t1 + bs - 1) / bs;
    const long long gmax = (long long)num_sms() * 32;
    if (g1 > gmax) g1 = gmax;
    c2s_ij_kernel<<<(int)g1, bs, 0, st>>>(cart, tmp, ncomp, nfc, naoc, npc, nfs, naos, ptr_i, idx_i, val_i, ptr,
                                          idx, val);
    int rc = check_launch("c2s_ij_kernel");
    if (rc) return rc;
    const long long t2 = rows * ((long long)naos * (naos + 1) / 2);
    long long g2 = (t2 + bs - 1) / bs;
    if (g2 > gmax) g2 = gmax;
    c2s_kl_kernel<<<(int)g2, bs, 0, st>>>(tmp, out, rows, npc, naos, ptr, idx, val);
    return check_launch("c2s_kl_kernel");
}

}  // extern "C"

// ---- Spherical transform for callers that cannot allocate device memory ----
//
// Some callers cannot call cudaMalloc: a host application that hands this
// library a device it has already carved up with its own pool allocator, or
// one that forbids allocation once its time step is running (cudaMalloc can
// synchronise the device and stall the work other components have queued).
// They can pass their input and output buffers but have nowhere to put the
// transform's intermediate.  This variant keeps that intermediate in a
// fixed, file-scope device array instead.
//   * The array holds kC2sScratchDoubles doubles (32 MiB).  Every GPU that
//     loads the library reserves it until the process exits.
//   * Host code cannot use the array's name as a device address, so the
//     first call on each device (with that device current) looks the address
//     up with cudaGetSymbolAddress and caches it.  Make that first call before
//     any stream capture.
//   * All calls share the one array.  Nothing in it has to start at zero:
//     the first pass writes every element the second pass reads.  Calls whose
//     work overlaps on the GPU (two streams, or several host threads) race on
//     the array and must be serialised by the caller.
static constexpr long long kC2sScratchDoubles = 4ll << 20;
static __device__ __align__(256) double g_c2s_scratch[kC2sScratchDoubles];

// The cached address belongs to the device's primary context, which this
// library assumes lives for the whole process (a cudaDeviceReset creates a new
// context with a new address; call nothing here after one).  First calls from
// several host threads may each look the address up; they store the same
// value, through an atomic, so the cache is free of data races.
static int c2s_scratch_address(double **out)
{
    static std::atomic<double *> addr[64];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        set_error("ccsd_b200_cart2sph_s2kl_noalloc: no current CUDA device");
        return CCSD_B200_ERR_LAUNCH;
    }
    double *a = addr[dev].load(std::memory_order_acquire);
    if (!a) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_c2s_scratch);
        if (e != cudaSuccess || !p) {
            set_error("ccsd_b200_cart2sph_s2kl_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            return CCSD_B200_ERR_LAUNCH;
        }
        a = static_cast<double *>(p);
        addr[dev].store(a, std::memory_order_release);
    }
    *out = a;
    return CCSD_B200_OK;
}

extern "C" int ccsd_b200_cart2sph_s2kl_noalloc(const double *cart, double *out, int ncomp, int nfc, int naoc,
                                               int nfs, int naos, const int32_t *ptr_i, const int32_t *idx_i,
                                               const double *val_i, const int32_t *ptr, const int32_t *idx,
                                               const double *val, void *stream)
{
    if (!cart || !out || ncomp <= 0 || nfc <= 0 || naoc <= 0 || nfs <= 0 || naos <= 0 || !ptr_i || !idx_i ||
        !val_i || !ptr || !idx || !val) {
        set_error("ccsd_b200_cart2sph_s2kl_noalloc: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    const long long npc = (long long)naoc * (naoc + 1) / 2;
    const long long rows = (long long)ncomp * nfs * naos;
    if (rows > kC2sScratchDoubles || npc > kC2sScratchDoubles / rows) {
        set_error("ccsd_b200_cart2sph_s2kl_noalloc: the block needs %lld doubles of scratch, the built-in "
                  "buffer holds %lld (32 MiB); split the i-shell range or use ccsd_b200_cart2sph_s2kl",
                  rows * npc, kC2sScratchDoubles);
        return CCSD_B200_ERR_ARG;
    }
    double *tmp = nullptr;
    int rc = c2s_scratch_address(&tmp);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int bs = 256;
    const long long gmax = (long long)num_sms() * 32;
    long long g1 = (rows * npc + bs - 1) / bs;
    if (g1 > gmax) g1 = gmax;
    c2s_ij_kernel<<<(int)g1, bs, 0, st>>>(cart, tmp, ncomp, nfc, naoc, npc, nfs, naos, ptr_i, idx_i, val_i, ptr,
                                          idx, val);
    if ((rc = check_launch("c2s_ij_kernel (no-alloc)"))) return rc;
    long long g2 = (rows * ((long long)naos * (naos + 1) / 2) + bs - 1) / bs;
    if (g2 > gmax) g2 = gmax;
    c2s_kl_kernel<<<(int)g2, bs, 0, st>>>(tmp, out, rows, npc, naos, ptr, idx, val);
    return check_launch("c2s_kl_kernel (no-alloc)");
}
