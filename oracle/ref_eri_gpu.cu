/*
 * ORACLE / COMPARATOR -- test and benchmark infrastructure only.
 *
 * Launcher that runs the reference's own ERI kernels on the GPU
 * (fill_int2e_kernel, ref: ccsd_gpu/cuda/int2e_module.py:130-463;
 *  fill_int2e_ip1_kernel, ref: ccsd_gpu/cuda/int2e_ip1_module.py:273-667),
 * compiled by nvcc for sm_100a, so that the package's ERI kernels can be timed
 * and checked beside the reference's GPU algorithm on the same device.  The
 * kernel sources are not in this repository: build_ref.py regenerates them
 * from the reference checkout (the reference's _build_cuda_source) into
 * oracle/_ref/ and compiles this file there into oracle/_ref/libref_eri_gpu.so.
 * Nothing in the package links or loads this library.
 *
 * The launch mirrors the reference's _compute_cart loop: one launch per
 * decontracted i-shell, grid = nbas * n_kl_pairs blocks of dim3(1, 32), and
 * the dynamic shared memory the reference sizes per i-shell
 * (ref: ccsd_gpu/cuda/int2e_gpu.py:78-106, ccsd_gpu/cuda/int2e_ip1_gpu.py:187-214):
 * 3 g-arrays of (li + 1 + deriv)(lmax + 1)^3 doubles, 2 * 9 Rys values and
 * iprim * max_prim contraction products.  The output block is zeroed first,
 * as the reference allocates it with cupy.zeros.
 */
#include <cuda_runtime.h>
#include <stdint.h>

namespace ref_int2e_gpu {
#include "int2e_src.inc"
}
namespace ref_ip1_gpu {
#include "int2e_ip1_src.inc"
}

extern "C" {

/*
 * Cartesian s2kl block of decontracted shells [dc_b0, dc_b1) x all j x all
 * k >= l into out ((3 if deriv) x nf x nao x nao(nao+1)/2, device).  atm,
 * bas, env, ao_loc and kl_pairs are device arrays; bas_host and ao_loc_host
 * are host copies of bas and ao_loc (the launch loop reads l, nprim and the
 * function offsets of each i-shell on the host, as the reference does).
 * Returns a cudaError_t value (0 = success).
 */
int ref_gpu_eri_cart(int deriv, double *out, const int32_t *atm, const int32_t *bas, const double *env,
                     const int32_t *ao_loc, const int32_t *bas_host, const int32_t *ao_loc_host, int dc_b0,
                     int dc_b1, int nbas, int nao, const int32_t *kl_pairs, int n_kl_pairs, int max_l,
                     int max_prim, void *stream)
{
    cudaStream_t st = (cudaStream_t)stream;
    const long long nao_pair = (long long)nao * (nao + 1) / 2;
    const int nf = ao_loc_host[dc_b1] - ao_loc_host[dc_b0];
    cudaError_t e = cudaMemsetAsync(out, 0, sizeof(double) * (deriv ? 3 : 1) * (long long)nf * nao * nao_pair, st);
    if (e != cudaSuccess) return (int)e;
    const dim3 block(1, 32);
    const long long grid = (long long)nbas * n_kl_pairs;
    const int l1 = max_l + 1;
    for (int ish = dc_b0; ish < dc_b1; ish++) {
        const int li = bas_host[ish * 8 + 1];
        const int iprim = bas_host[ish * 8 + 2];
        const int fi_offset = ao_loc_host[ish] - ao_loc_host[dc_b0];
        const long long g = (long long)(li + 1 + (deriv ? 1 : 0)) * l1 * l1 * l1;
        const size_t smem = (size_t)(3 * g + 2 * 9 + (long long)iprim * max_prim) * sizeof(double);
        if (deriv)
            ref_ip1_gpu::fill_int2e_ip1_kernel<<<(unsigned)grid, block, smem, st>>>(
                out, atm, bas, env, ao_loc, ish, fi_offset, nf, nbas, nao, (int)nao_pair, kl_pairs, n_kl_pairs);
        else
            ref_int2e_gpu::fill_int2e_kernel<<<(unsigned)grid, block, smem, st>>>(
                out, atm, bas, env, ao_loc, ish, fi_offset, nf, nbas, nao, (int)nao_pair, kl_pairs, n_kl_pairs);
        e = cudaGetLastError();
        if (e != cudaSuccess) return (int)e;
    }
    return 0;
}

}
