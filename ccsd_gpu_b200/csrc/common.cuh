// Shared definitions for the ccsd_b200 CUDA sources.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

// libcint / PySCF slot layout of _atm and _bas rows
#define CB_ATM_SLOTS 6
#define CB_PTR_COORD 1
#define CB_BAS_SLOTS 8
#define CB_ATOM_OF 0
#define CB_ANG_OF 1
#define CB_NPRIM_OF 2
#define CB_NCTR_OF 3
#define CB_PTR_EXP 5
#define CB_PTR_COEFF 6

#define CB_LMAX 4

// status codes returned by every extern "C" entry point
#define CCSD_B200_OK 0
#define CCSD_B200_ERR_ARG 1
#define CCSD_B200_ERR_LAUNCH 2
#define CCSD_B200_ERR_TIMEOUT 3
#define CCSD_B200_ERR_NONFINITE 4
#define CCSD_B200_ERR_UNSUPPORTED 5

namespace cb {

void set_error(const char *fmt, ...);
int check_launch(const char *what);

__host__ __device__ __forceinline__ int ncart(int l) { return (l + 1) * (l + 2) / 2; }

// pair index p = k (k + 1) / 2 + l (k >= l) -> (k, l)
__device__ __forceinline__ void decode_pair(long long p, int &k, int &l)
{
    int kk = (int)((sqrt(8.0 * (double)p + 1.0) - 1.0) * 0.5);
    while ((long long)kk * (kk + 1) / 2 > p) kk--;
    while ((long long)(kk + 1) * (kk + 2) / 2 <= p) kk++;
    k = kk;
    l = (int)(p - (long long)kk * (kk + 1) / 2);
}

}  // namespace cb
