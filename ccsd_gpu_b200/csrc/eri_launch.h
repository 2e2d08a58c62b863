// Launchers of the ERI kernels (eri_kernels.cuh), instantiated per
// (derivative order D, LOW = all shells l <= 2) in the eri_inst_*.cu units.
#pragma once
#include <cuda_runtime.h>
#include <stddef.h>

namespace cb {

static constexpr int kWarps = 4;          // warps (quartets in flight) per CTA of the warp kernels (default)
static constexpr int kHeavyThreads = 256; // threads of the CTA (heavy-quartet) kernels
static constexpr int kMaxSlots = 64;      // slots per batch cap (warp kernels, per-output CTA path)
// slots per batch cap of the contracted-HRR path on a 256-thread CTA: one
// slot per thread in phase A, three (slot, direction) items per thread in B
// (measured against 64: heavy int2e_ip1 quartets of the benchmark list 11.0
// -> 10.75 ms, int2e 3.76 -> 3.56 ms)
static constexpr int kMaxSlotsCta = 256;
static constexpr int kParStride = 13;     // doubles of per-slot parameters (odd: lanes spread over banks)
static constexpr int kHcSmem = 3072;      // doubles of shared memory per warp on the l <= 2 kernels
static constexpr int kWarpCtas = 2;       // 4-warp CTAs resident per SM (255 registers, kHcSmem doubles per warp)

// Quartets whose Cartesian block has more functions than heavy_nf(D) go to
// the CTA-cooperative kernel; smaller ones are one warp each.  Measured on the
// 2^18-quartet benchmark set: int2e is fastest with the (dd|dp)-class blocks
// (648 functions) on warps, int2e_ip1 with them on CTAs (119 -> 89 ms).
static constexpr int kHeavyNf = 1000;
static constexpr int kHeavyNfIp1 = 500;
__host__ __device__ constexpr int heavy_nf(int D) { return D ? kHeavyNfIp1 : kHeavyNf; }

// MODE_S2KL_SPH: the s2kl block in spherical functions (l <= 2 kernels), a
// mode of its own so the Cartesian s2kl kernels carry no staging code
enum { MODE_S2KL = 0, MODE_QSUM = 1, MODE_GRAD = 2, MODE_FULL = 3, MODE_S2KL_SPH = 4 };

// Warps per CTA of the warp kernel of an epilogue mode.  The molecular lists
// (the gradient's ip1-Gamma contraction, the SCF's dense ERI tensor) run
// 8-warp CTAs, one per SM: every warp of an SM then walks the same part of the
// class-sorted list and shares one instruction working set (the kernels stall
// mostly on instruction fetch; measured 11-13% faster on (H2O)n/cc-pVDZ
// gradient lists, 7-11% on int2e).  The synthetic checksum list and the s2kl
// blocks keep 4-warp CTAs, two per SM (the checksum list ran 19% slower with 8).
__host__ __device__ constexpr int warps_of(int mode) { return mode == MODE_GRAD || mode == MODE_FULL ? 8 : kWarps; }

// Per-L-class choice of the warp kernels' accumulation path, over the 81
// classes (li, lj, lk, ll), l <= 2, in the quartet's own shell order, class
// id li*27 + lj*9 + lk*3 + ll: bit set in hc = contracted-HRR path whenever
// it fits, bit set in po = per-output path; neither = the measured rule.
// Passed to the kernels by value (kernel parameter space).
struct PathTable {
    unsigned long long hc[2] = {0ull, 0ull}, po[2] = {0ull, 0ull};

    __host__ __device__ int force(int li, int lj, int lk, int ll) const
    {
        if (li > 2 || lj > 2 || lk > 2 || ll > 2) return 0;
        const int c = li * 27 + lj * 9 + lk * 3 + ll;
        const unsigned long long bit = 1ull << (c & 63);
        if (hc[c >> 6] & bit) return 1;
        if (po[c >> 6] & bit) return 2;
        return 0;
    }
};

struct EriArgs {
    const int *atm = nullptr, *bas = nullptr;
    const double *env = nullptr;
    const int *ao_loc = nullptr;
    int ish0 = 0, ish1 = 0, nbas = 0, nao = 0;    // s2kl block
    double *out = nullptr;                         // s2kl output
    const int4 *quartets = nullptr;                // explicit list (or the s2kl heavy list)
    long long nq = 0;
    double *qsum = nullptr;                        // per-quartet checksums / gradient values
    const double *gamma = nullptr;                 // MODE_GRAD density
    int grow0 = 0, grows = 0;                      // MODE_GRAD: rows of gamma held (grows 0: all nao)
    double *full = nullptr;                        // MODE_FULL dense tensor
    int heavy = 0;                                 // heavy-quartet threshold (0: compiled default)
    int smem_warp = 0, smem_heavy = 0;             // doubles of shared memory per warp / per heavy CTA
    PathTable paths;                               // accumulation path per L-class (warp kernels)
    const int *ao_sph = nullptr;                   // s2kl, spherical output: AO offsets per shell
    const double *c2s = nullptr;                   //   and the d-shell cart->sph factors (5 x 6)
};

template <int D, bool LOW> int launch_s2kl(const EriArgs &a, long long grid, size_t smem, cudaStream_t st);
template <int D, bool LOW> int launch_s2kl_heavy(const EriArgs &a, long long grid, size_t smem, cudaStream_t st);
template <int D, bool LOW, int MODE> int launch_list(const EriArgs &a, long long grid, size_t smem, cudaStream_t st);
template <int D, bool LOW, int MODE>
int launch_list_heavy(const EriArgs &a, long long grid, size_t smem, cudaStream_t st);

}  // namespace cb
