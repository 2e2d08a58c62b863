/*
 * ORACLE -- test infrastructure only.
 *
 * Host-side shim that compiles the reference's own ERI kernels
 * (fill_int2e_kernel, ref: ccsd_gpu/cuda/int2e_module.py:130-463;
 *  fill_int2e_ip1_kernel, ref: ccsd_gpu/cuda/int2e_ip1_module.py:273-667)
 * as plain C++ for the CPU.  The kernel sources are not in this repository:
 * build_ref.py regenerates them from the reference checkout with the
 * reference's own _build_cuda_source() into oracle/_ref/ and compiles this
 * file there.  Every loop of those kernels is strided by blockDim.y, so
 * running one "thread" per block (blockDim.y = 1, __syncthreads a no-op)
 * executes the identical arithmetic serially.  Blocks run in parallel with
 * OpenMP; each block writes a disjoint set of output elements.
 */
#include <cmath>
#include <cstring>
#include <cstdio>

struct ref_dim3 { int x, y, z; };
static thread_local ref_dim3 threadIdx = {0, 0, 0};
static thread_local ref_dim3 blockIdx = {0, 0, 0};
static const ref_dim3 blockDim = {1, 1, 1};
#define __global__
#define __device__
#define __restrict__
#define __shared__ thread_local
static inline void __syncthreads() {}
using std::exp;
using std::sqrt;
using std::erf;

#define REF_SHM_DOUBLES (1 << 15)

namespace ref_int2e {
#include "int2e_src.inc"
thread_local double shm[REF_SHM_DOUBLES];
}
namespace ref_ip1 {
#include "int2e_ip1_src.inc"
thread_local double shm[REF_SHM_DOUBLES];
}

extern "C" {

/* Mirrors the launch loop of _compute_cart (ref: ccsd_gpu/cuda/int2e_gpu.py:81-106,
 * ccsd_gpu/cuda/int2e_ip1_gpu.py:190-214) for decontracted shells dc_b0..dc_b1. */
int ref_eri_cart(int deriv, double *out, const int *atm, const int *bas, const double *env,
                 const int *ao_loc, int dc_b0, int dc_b1, int nbas, int nao,
                 const int *kl_pairs, int n_kl_pairs)
{
    const long nao_pair = (long)nao * (nao + 1) / 2;
    const int nf = ao_loc[dc_b1] - ao_loc[dc_b0];
    memset(out, 0, sizeof(double) * (deriv ? 3 : 1) * (long)nf * nao * nao_pair);
    for (int ish = dc_b0; ish < dc_b1; ish++) {
        const int fi_offset = ao_loc[ish] - ao_loc[dc_b0];
        const long nblocks = (long)nbas * n_kl_pairs;
#pragma omp parallel for schedule(dynamic, 4)
        for (long b = 0; b < nblocks; b++) {
            blockIdx.x = (int)b;
            if (deriv)
                ref_ip1::fill_int2e_ip1_kernel(out, atm, bas, env, ao_loc, ish, fi_offset, nf,
                                               nbas, nao, (int)nao_pair, kl_pairs, n_kl_pairs);
            else
                ref_int2e::fill_int2e_kernel(out, atm, bas, env, ao_loc, ish, fi_offset, nf,
                                             nbas, nao, (int)nao_pair, kl_pairs, n_kl_pairs);
        }
    }
    return 0;
}

/* Rys roots/weights of the reference (rys_roots_simple). */
void ref_rys_roots(int nroots, double x, double *r, double *w)
{
    ref_int2e::rys_roots_simple(nroots, x, r, w);
}

}

extern "C" {
/*
 * Per-quartet run of the reference kernels: each quartet (i, j, k, l) of an
 * explicit list is presented to the reference kernel as a 4-shell basis
 * (local shells i, j, l, k = 0..3, one kl pair (3, 2) so that the packed kl
 * index has k >= l, block index 1 -> jsh = 1), its
 * Cartesian block is read back and reduced to the two checksums of
 * ccsd_b200_eri_quartet_checksums.  Shells must be decontracted (nctr == 1).
 */
int ref_eri_quartet_checksums(int deriv, const int *atm, const int *bas, const double *env,
                              const int *quartets, long nq, double *qsum)
{
    const int ncomp = deriv ? 3 : 1;
#pragma omp parallel for schedule(dynamic, 16)
    for (long q = 0; q < nq; q++) {
        int lbas[4 * 8], ao_loc[5], l[4], nfs[4];
        ao_loc[0] = 0;
        const int order[4] = {0, 1, 3, 2};   /* local slot -> quartet position */
        for (int s = 0; s < 4; s++) {
            memcpy(lbas + 8 * s, bas + 8 * quartets[4 * q + order[s]], 8 * sizeof(int));
            l[s] = lbas[8 * s + 1];
            nfs[s] = (l[s] + 1) * (l[s] + 2) / 2;
            ao_loc[s + 1] = ao_loc[s] + nfs[s];
        }
        const int nao = ao_loc[4], npair = nao * (nao + 1) / 2;
        const int kl_pairs[2] = {3, 2};
        double *buf = new double[(long)ncomp * nfs[0] * nao * npair];
        blockIdx.x = 1;
        if (deriv)
            ref_ip1::fill_int2e_ip1_kernel(buf, atm, lbas, env, ao_loc, 0, 0, nfs[0], 4, nao, npair, kl_pairs, 1);
        else
            ref_int2e::fill_int2e_kernel(buf, atm, lbas, env, ao_loc, 0, 0, nfs[0], 4, nao, npair, kl_pairs, 1);
        for (int c = 0; c < ncomp; c++) {
            double s1 = 0, s2 = 0;
            int f = 0;
            for (int fi = 0; fi < nfs[0]; fi++)
                for (int fj = 0; fj < nfs[1]; fj++)
                    for (int fk = 0; fk < nfs[3]; fk++)
                        for (int fl = 0; fl < nfs[2]; fl++, f++) {
                            const long k = ao_loc[3] + fk, ll = ao_loc[2] + fl;
                            const double v = buf[(((long)c * nfs[0] + fi) * nao + ao_loc[1] + fj) * npair + k * (k + 1) / 2 + ll];
                            s1 += v * (1.0 + 0.125 * (f & 7));
                            s2 += v * v;
                        }
            qsum[(q * ncomp + c) * 2] = s1;
            qsum[(q * ncomp + c) * 2 + 1] = s2;
        }
        delete[] buf;
    }
    return 0;
}
}
