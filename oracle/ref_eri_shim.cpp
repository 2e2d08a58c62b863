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
