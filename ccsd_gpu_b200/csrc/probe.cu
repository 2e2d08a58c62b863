// FP64 FMA throughput probe: the FP64-pipe roofline denominator for the ERI
// kernels (the driver-measured peaks cover HBM and bf16 tensor throughput only).
#include "common.cuh"

namespace cb {

// 8 independent FMA chains per thread; every result feeds the output so
// nothing is eliminated.  FLOPs = 2 * 8 * iters * threads.
__global__ void __launch_bounds__(256) fp64_fma_probe_kernel(double *out, int iters, double a, double b)
{
    double x[8];
#pragma unroll
    for (int k = 0; k < 8; k++) x[k] = threadIdx.x * 1e-3 + k;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int k = 0; k < 8; k++) x[k] = fma(x[k], a, b);
    }
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < 8; k++) s += x[k];
    if (s == 1.2345e-300) out[blockIdx.x * blockDim.x + threadIdx.x] = s;   // practically never stored
}

}  // namespace cb

extern "C" int ccsd_b200_fp64_fma_probe(double *out, int blocks, int iters, void *stream)
{
    if (!out || blocks <= 0 || iters <= 0) {
        cb::set_error("ccsd_b200_fp64_fma_probe: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    cb::fp64_fma_probe_kernel<<<blocks, 256, 0, (cudaStream_t)stream>>>(out, iters, 0.999999999, 1e-9);
    return cb::check_launch("fp64_fma_probe_kernel");
}
