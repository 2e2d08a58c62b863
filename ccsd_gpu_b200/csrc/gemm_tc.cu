// Split-precision tensor-core GEMM for sm_100a (tcgen05 + TMA + TMEM).
//
//   D[m, n] = sum_k A[m, k] B[n, k]     (A, B given in FP64)
// is evaluated as  A_hi B_hi + A_hi B_lo + A_lo B_hi  with A = A_hi + A_lo,
// B = B_hi + B_lo split into two TF32 (kind::tf32) or BF16 (kind::f16) parts:
// three tcgen05.mma per K step into an FP32 accumulator in tensor memory.
// The TF32 split represents an FP64 value to ~2^-24 relative, so the error is
// set by the FP32 accumulation; to keep it at the FP32 level for long K, the
// accumulator is drained into the FP64 output every 512 k (double-buffered in
// TMEM, so the MMAs of chunk c+1 overlap the drain of chunk c).  The drain
// scatters through per-row / per-column offset tables, so any einsum output
// permutation is written in place:  out[off_m[m] + off_n[n]] = alpha*D + beta*out.
//
// Operands are produced by split_pack_kernel: it gathers an FP64 operand (up
// to two linear terms, each addressed through offset tables, so transposes and
// "2 t - t^T" combinations fuse into the pack), splits every value into hi and
// lo parts and writes K-major [rows_pad x k_pad] arrays for TMA (k_pad: K
// rounded up to a 16-byte row; the values past K are zero).  Rows past the
// array and k past k_pad are not stored: TMA fills the out-of-bounds part of
// a 128 x 128-byte box with zeros, so skinny operands (24 rows, or K = 24)
// cost only their own bytes.
//
// CTA = 320 threads, one 128 x 128 output tile:
//   warp 0      TMA producer (lane 0) into a 3-stage ring of {A_hi, A_lo, B_hi,
//               B_lo} tiles (128 rows x 128 B, 128 B swizzle); owns TMEM alloc.
//   warp 1      MMA issuer (lane 0); commits stage releases and chunk-ready.
//   warps 2..9  drain TMEM: warp w reads lanes 32*(w%4) .. +31, columns
//               64*((w-2)/4) .. +63, and keeps its 32 x 64 block as FP64
//               running sums in registers across all k chunks; the output is
//               written once, after the last chunk.
// Every mbarrier wait is bounded by the global timer (2 s): on expiry the
// thread records a code in `status` and leaves its loop -- no trap, no
// unbounded spin.
#include "common.cuh"

#include <algorithm>

#include <cuda.h>
#include <cudaTypedefs.h>
#include <cuda_bf16.h>

namespace cb {

static constexpr int TC_BM = 128;
static constexpr int TC_BN = 128;
static constexpr int TC_STAGES = 3;
static constexpr int TC_ROWB = 128;                      // bytes per tile row (swizzle span)
static constexpr int TC_TILE_BYTES = TC_BM * TC_ROWB;    // 16 KiB
static constexpr int TC_STAGE_BYTES = 4 * TC_TILE_BYTES;
static constexpr int TC_DRAIN_WARPS = 8;                // 2 per TMEM lane quadrant
static constexpr int TC_THREADS = 64 + 32 * TC_DRAIN_WARPS;
static constexpr int TC_CHUNK_K = 512;                   // k per FP32 accumulation chunk
static constexpr int TC_GROUP_M = 8;                     // row tiles per raster group
static constexpr int TC_EPI_LD = 65;                     // epilogue staging row stride (doubles)
static_assert(TC_DRAIN_WARPS * 32 * TC_EPI_LD * 8 <= TC_STAGES * TC_STAGE_BYTES, "epilogue staging fits the ring");
static constexpr unsigned long long TC_WAIT_NS = 2000000000ull;

enum { KIND_TF32 = 0, KIND_BF16 = 1 };

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ unsigned long long global_ns()
{
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// bounded wait: false (and `code` recorded in *status) after `limit_ns`
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, int *status, int code,
                                          unsigned long long limit_ns = TC_WAIT_NS)
{
    const unsigned long long t0 = global_ns();
    for (unsigned it = 0;; it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63) == 63) {
            if (*(volatile int *)status != 0) return false;       // another CTA already gave up
            if (global_ns() - t0 > limit_ns) break;
        }
    }
    atomicCAS(status, 0, code);
    return false;
}

// Bounded wait used on the abort path only: waits for the asynchronous work
// this thread has already issued (TMA loads, tcgen05.mma) to land, whatever
// other CTAs recorded in `status`.  Returns false after `limit_ns`.
__device__ __forceinline__ bool mbar_settle(uint64_t *bar, uint32_t parity, unsigned long long limit_ns = TC_WAIT_NS)
{
    const unsigned long long t0 = global_ns();
    for (unsigned it = 0;; it++) {
        if (mbar_try_wait(bar, parity)) return true;
        if ((it & 63) == 63 && global_ns() - t0 > limit_ns) return false;
    }
}

__device__ __forceinline__ void mbar_arrive(uint64_t *bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ void tma_load_2d(const CUtensorMap *map, uint64_t *bar, void *dst, int x, int y)
{
    asm volatile(
        "cp.async.bulk.tensor.2d.shared::cta.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];"
        ::"r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
        : "memory");
}

// K-major, 128 B swizzle UMMA shared-memory descriptor (8-row groups 1024 B apart)
__device__ __forceinline__ uint64_t umma_desc(uint32_t saddr)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr >> 4) & 0x3FFF);          // start address
    d |= (uint64_t)1 << 16;                            // leading byte offset (unused for SW128 K-major)
    d |= (uint64_t)(1024 >> 4) << 32;                  // stride byte offset
    d |= (uint64_t)1 << 46;                            // descriptor version (sm_100)
    d |= (uint64_t)2 << 61;                            // SWIZZLE_128B
    return d;
}

template <int KIND>
__device__ __forceinline__ uint32_t instr_desc()
{
    const uint32_t fmt = KIND == KIND_TF32 ? 2u : 1u;  // A/B format: TF32 = 2, BF16 = 1
    return (1u << 4)                                   // D format F32
           | (fmt << 7) | (fmt << 10)                  // A, B formats, both K-major
           | ((uint32_t)(TC_BN >> 3) << 17)            // N
           | ((uint32_t)(TC_BM >> 4) << 24);           // M
}

template <int KIND>
__device__ __forceinline__ void umma(uint32_t tmem_d, uint64_t da, uint64_t db, uint32_t idesc, uint32_t acc)
{
    if (KIND == KIND_TF32)
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
    else
        asm volatile(
            "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}"
            ::"r"(tmem_d), "l"(da), "l"(db), "r"(idesc), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

__device__ __forceinline__ void umma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                 ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, "
        "%14, %15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; i++) v[i] = __uint_as_float(r[i]);
}

template <int KIND>
__global__ void __launch_bounds__(TC_THREADS, 1) tc_split_gemm_kernel(
    const __grid_constant__ CUtensorMap map_ahi, const __grid_constant__ CUtensorMap map_alo,
    const __grid_constant__ CUtensorMap map_bhi, const __grid_constant__ CUtensorMap map_blo,
    int M, int N, int mtiles, int ntiles, int kblocks, int kb_per_split, double *__restrict__ out,
    const long long *__restrict__ off_m, const long long *__restrict__ off_n, double alpha, double beta,
    double *__restrict__ partial, int *__restrict__ status)
{
    extern __shared__ __align__(1024) uint8_t smem_raw[];
    uint8_t *smem = reinterpret_cast<uint8_t *>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    __shared__ __align__(8) uint64_t full_bar[TC_STAGES], empty_bar[TC_STAGES], accf_bar[2], acce_bar[2];
    __shared__ uint32_t tmem_base_s;
    __shared__ int abort_s;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // A wait already expired in this or an earlier GEMM (the status is sticky
    // until the host reads it): leave before any TMEM allocation or TMA, with
    // the outputs untouched.  The decision is made once for the whole CTA.
    if (threadIdx.x == 0) abort_s = *(volatile int *)status;
    __syncthreads();
    if (abort_s) return;
    // raster: groups of TC_GROUP_M row tiles, row tile fastest inside a group, so
    // the CTAs resident at one time share a few A row tiles and each B tile is
    // fetched from HBM about once
    // (split-K: block = split * tiles + tile; split s covers k blocks
    // [s * kb_per_split, min(kblocks, (s + 1) * kb_per_split)) and writes its
    // FP64 partial tile to partial[s][M][N] for splitk_reduce_kernel)
    const int tiles = mtiles * ntiles;
    const int split = blockIdx.x / tiles;
    const int tile = blockIdx.x - split * tiles;
    const int group = tile / (TC_GROUP_M * ntiles);
    const int first_m = group * TC_GROUP_M;
    const int gsize = min(mtiles - first_m, TC_GROUP_M);
    const int local = tile - group * TC_GROUP_M * ntiles;
    const int m0 = (first_m + local % gsize) * TC_BM, n0 = (local / gsize) * TC_BN;
    const int kb_begin = split * kb_per_split;
    const int nkb = min(kblocks - kb_begin, kb_per_split);
    constexpr int KB_ELEMS = TC_ROWB / (KIND == KIND_TF32 ? 4 : 2);   // k per pipeline stage
    constexpr int KB_PER_CHUNK = TC_CHUNK_K / KB_ELEMS;
    const int nchunks = (nkb + KB_PER_CHUNK - 1) / KB_PER_CHUNK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < TC_STAGES; s++) {
            mbar_init(&full_bar[s], 1);
            mbar_init(&empty_bar[s], 1);
        }
        for (int b = 0; b < 2; b++) {
            mbar_init(&accf_bar[b], 1);
            mbar_init(&acce_bar[b], TC_DRAIN_WARPS);
        }
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                     ::"r"(smem_u32(&tmem_base_s)), "r"(2 * TC_BN));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t tmem = tmem_base_s;

    if (warp == 0) {
        if (lane == 0) {
            // ---- TMA producer
            int issued = 0;
            for (int kb = 0; kb < nkb; kb++) {
                const int s = kb % TC_STAGES;
                const uint32_t ph = (kb / TC_STAGES) & 1;
                if (!mbar_wait(&empty_bar[s], ph ^ 1, status, 1)) break;
                uint8_t *st = smem + s * TC_STAGE_BYTES;
                mbar_expect_tx(&full_bar[s], TC_STAGE_BYTES);
                const int kx = (kb_begin + kb) * KB_ELEMS;
                tma_load_2d(&map_ahi, &full_bar[s], st, kx, m0);
                tma_load_2d(&map_alo, &full_bar[s], st + TC_TILE_BYTES, kx, m0);
                tma_load_2d(&map_bhi, &full_bar[s], st + 2 * TC_TILE_BYTES, kx, n0);
                tma_load_2d(&map_blo, &full_bar[s], st + 3 * TC_TILE_BYTES, kx, n0);
                issued = kb + 1;
            }
            // The last TC_STAGES loads may not have been consumed (abort, or the
            // normal end): the CTA must not exit with bulk copies in flight into
            // its shared memory, so wait (bounded) until each of them has landed.
            for (int kb = issued > TC_STAGES ? issued - TC_STAGES : 0; kb < issued; kb++)
                mbar_settle(&full_bar[kb % TC_STAGES], (kb / TC_STAGES) & 1);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            // ---- MMA issuer
            const uint32_t idesc = instr_desc<KIND>();
            bool ok = true;
            int last = -1;                          // chunk of the last accf commit
            for (int c = 0; c < nchunks && ok; c++) {
                const int buf = c & 1;
                const uint32_t use = (uint32_t)(c >> 1);
                if (!mbar_wait(&acce_bar[buf], (use & 1) ^ 1, status, 2)) break;
                asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                const uint32_t acc_tmem = tmem + buf * TC_BN;
                const int kb0 = c * KB_PER_CHUNK, kb1 = min(nkb, kb0 + KB_PER_CHUNK);
                for (int kb = kb0; kb < kb1; kb++) {
                    const int s = kb % TC_STAGES;
                    const uint32_t ph = (kb / TC_STAGES) & 1;
                    if (!mbar_wait(&full_bar[s], ph, status, 3)) { ok = false; break; }
                    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                    const uint32_t base = smem_u32(smem + s * TC_STAGE_BYTES);
#pragma unroll
                    for (int k = 0; k < 4; k++) {          // 128 B row = 4 UMMA K steps of 32 B
                        const uint64_t ahi = umma_desc(base + k * 32);
                        const uint64_t alo = umma_desc(base + TC_TILE_BYTES + k * 32);
                        const uint64_t bhi = umma_desc(base + 2 * TC_TILE_BYTES + k * 32);
                        const uint64_t blo = umma_desc(base + 3 * TC_TILE_BYTES + k * 32);
                        umma<KIND>(acc_tmem, ahi, bhi, idesc, (kb != kb0 || k) ? 1u : 0u);
                        umma<KIND>(acc_tmem, ahi, blo, idesc, 1u);
                        umma<KIND>(acc_tmem, alo, bhi, idesc, 1u);
                    }
                    umma_commit(&empty_bar[s]);     // stage reusable once these MMAs finish
                }
                umma_commit(&accf_bar[buf]);        // chunk accumulated (also on the error path)
                last = c;
            }
            // TMEM is freed at the end of the kernel: every MMA issued here must
            // have completed first.  The last commit tracks all of them.
            if (last >= 0) mbar_settle(&accf_bar[last & 1], ((uint32_t)(last >> 1)) & 1);
        }
    } else {
        // ---- drain warps: FP64 running sums in registers, one write at the end
        //      (lane = output row of the TMEM lane quadrant q)
        const int q = warp & 3;
        const int cbase = 64 * ((warp - 2) >> 2);
        double sum[64];
#pragma unroll
        for (int i = 0; i < 64; i++) sum[i] = 0.0;
        bool ok = true;
        for (int c = 0; c < nchunks; c++) {
            const int buf = c & 1;
            const uint32_t use = (uint32_t)(c >> 1);
            const bool got = mbar_wait(&accf_bar[buf], use & 1, status, 4);
            asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
            // warp-uniform: tcgen05.ld is a .sync.aligned instruction
            if (!__all_sync(0xffffffffu, got && *(volatile int *)status == 0)) { ok = false; break; }
#pragma unroll
            for (int c0 = 0; c0 < 64; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + buf * TC_BN + ((uint32_t)(q * 32) << 16) + cbase + c0, v);
#pragma unroll
                for (int i = 0; i < 16; i++) sum[c0 + i] += (double)v[i];
            }
            asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
            __syncwarp();
            if (lane == 0) mbar_arrive(&acce_bar[buf]);
        }
        // Epilogue through shared memory: once the last chunk has been read,
        // every MMA of this tile has completed, so the stage ring is free.  Each
        // warp stores its 32 x 64 block row-major (stride 65: conflict-free in
        // both directions) and writes it back one output row at a time, lanes
        // along n: coalesced whenever off_n is contiguous.
        if (ok) {
            double *blk = reinterpret_cast<double *>(smem) + (warp - 2) * (32 * TC_EPI_LD);
#pragma unroll
            for (int i = 0; i < 64; i++) blk[lane * TC_EPI_LD + i] = sum[i];
            __syncwarp();
            const int mrow0 = m0 + q * 32;
            for (int r = 0; r < 32 && mrow0 + r < M; r++) {
                const int mr = mrow0 + r;
                const long long om = partial ? 0 : off_m[mr];
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int c = lane + 32 * h;
                    const int n = n0 + cbase + c;
                    if (n >= N) continue;
                    const double v = blk[r * TC_EPI_LD + c];
                    if (partial) {
                        partial[((size_t)split * M + mr) * N + n] = v;
                    } else {
                        double *o = out + om + off_n[n];
                        *o = beta == 0.0 ? alpha * v : fma(beta, *o, alpha * v);
                    }
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    if (warp == 0) {
        asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * TC_BN));
    }
}

// ---- failure-path probe: the pipeline's bounded mbarrier wait on a barrier
// that nothing arrives at.  The wait gives up after `limit_ns`, records
// `code` in *status and the kernel returns normally (no trap), so the host
// sees the error and the context stays usable.
__global__ void wait_probe_kernel(int *__restrict__ status, unsigned long long limit_ns, int code)
{
    __shared__ __align__(8) uint64_t bar;
    if (threadIdx.x == 0) {
        mbar_init(&bar, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        mbar_wait(&bar, 0, status, code, limit_ns);     // phase 0 never completes
    }
}

// ---- split-K reduction: out = alpha * sum_s partial[s] + beta * out (fixed order) ----
__global__ void splitk_reduce_kernel(const double *__restrict__ partial, int ksplit, int M, int N,
                                     double *__restrict__ out, const long long *__restrict__ off_m,
                                     const long long *__restrict__ off_n, double alpha, double beta)
{
    const long long mn = (long long)M * N;
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < mn;
         e += (long long)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int s = 0; s < ksplit; s++) acc += partial[s * mn + e];
        const int m = (int)(e / N), n = (int)(e - (long long)m * N);
        double *o = out + off_m[m] + off_n[n];
        *o = beta == 0.0 ? alpha * acc : fma(beta, *o, alpha * acc);
    }
}

// ---- operand gather + split ----
// dst row r, column k  <-  c1 * src1[o1r[r] + o1k[k]] + c2 * src2[o2r[r] + o2k[k]]
// (second term optional), split into hi + lo of the MMA input type.
template <int KIND>
__device__ __forceinline__ void split_store(void *__restrict__ hi, void *__restrict__ lo, long long e, double x)
{
    if (KIND == KIND_TF32) {
        uint32_t h, l;
        const float xf = (float)x;
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(xf));
        const float rest = (float)(x - (double)__uint_as_float(h));
        asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(rest));
        reinterpret_cast<uint32_t *>(hi)[e] = h;
        reinterpret_cast<uint32_t *>(lo)[e] = l;
    } else {
        const __nv_bfloat16 h = __double2bfloat16(x);
        const __nv_bfloat16 l = __double2bfloat16(x - (double)__bfloat162float(h));
        reinterpret_cast<__nv_bfloat16 *>(hi)[e] = h;
        reinterpret_cast<__nv_bfloat16 *>(lo)[e] = l;
    }
}

__device__ __forceinline__ double pack_value(const double *__restrict__ src1, const long long *__restrict__ o1r,
                                             const long long *__restrict__ o1k, double c1,
                                             const double *__restrict__ src2, const long long *__restrict__ o2r,
                                             const long long *__restrict__ o2k, double c2, int r, int k, int rows,
                                             int K)
{
    if (r >= rows || k >= K) return 0.0;
    double x = c1 * src1[o1r[r] + o1k[k]];
    if (src2) x = fma(c2, src2[o2r[r] + o2k[k]], x);
    return x;
}

// 32 x 32 tiles, 32 x 8 threads.  The packed array is K-major, so writes go
// with lanes along k.  ROWFAST: the source is contiguous along the packed
// rows (a transposing gather), so lanes read along rows and the tile turns
// through shared memory; otherwise lanes read and write along k directly.
template <int KIND, bool ROWFAST>
__global__ void __launch_bounds__(256) split_pack_kernel(
    const double *__restrict__ src1, const long long *__restrict__ o1r, const long long *__restrict__ o1k, double c1,
    const double *__restrict__ src2, const long long *__restrict__ o2r, const long long *__restrict__ o2k, double c2,
    int rows, int K, int rows_pad, int k_pad, void *__restrict__ hi, void *__restrict__ lo)
{
    __shared__ double tile[32][33];
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
    const int k0 = blockIdx.x * 32;
    const int nrt = (rows_pad + 31) / 32;
    for (int rt = blockIdx.y; rt < nrt; rt += gridDim.y) {
        const int r0 = rt * 32;
        if (ROWFAST) {
#pragma unroll
            for (int i = 0; i < 4; i++)
                tile[ty + 8 * i][tx] = pack_value(src1, o1r, o1k, c1, src2, o2r, o2k, c2, r0 + tx, k0 + ty + 8 * i,
                                                  rows, K);
            __syncthreads();
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int r = r0 + ty + 8 * i, k = k0 + tx;
                if (r < rows_pad && k < k_pad) split_store<KIND>(hi, lo, (long long)r * k_pad + k, tile[tx][ty + 8 * i]);
            }
            __syncthreads();
        } else {
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const int r = r0 + ty + 8 * i, k = k0 + tx;
                if (r < rows_pad && k < k_pad)
                    split_store<KIND>(hi, lo, (long long)r * k_pad + k,
                                      pack_value(src1, o1r, o1k, c1, src2, o2r, o2k, c2, r, k, rows, K));
            }
        }
    }
}

// ---- host side ----
static PFN_cuTensorMapEncodeTiled_v12000 get_encode()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    if (!fn) {
        cudaDriverEntryPointQueryResult q;
        void *p = nullptr;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

static int make_map(CUtensorMap *map, const void *base, int kind, int rows_pad, int k_pad)
{
    auto enc = get_encode();
    if (!enc) {
        set_error("cuTensorMapEncodeTiled unavailable");
        return CCSD_B200_ERR_LAUNCH;
    }
    const int esz = kind == KIND_TF32 ? 4 : 2;
    cuuint64_t dims[2] = {(cuuint64_t)k_pad, (cuuint64_t)rows_pad};
    cuuint64_t strides[1] = {(cuuint64_t)k_pad * esz};
    cuuint32_t box[2] = {(cuuint32_t)(TC_ROWB / esz), (cuuint32_t)TC_BM};
    cuuint32_t estr[2] = {1, 1};
    CUresult r = enc(map, kind == KIND_TF32 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2,
                     const_cast<void *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                     CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                     CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("cuTensorMapEncodeTiled failed (%d)", (int)r);
        return CCSD_B200_ERR_LAUNCH;
    }
    return CCSD_B200_OK;
}

template <int KIND>
static int launch_tc(const CUtensorMap &ma, const CUtensorMap &mal, const CUtensorMap &mb, const CUtensorMap &mbl,
                     int M, int N, int m_pad, int n_pad, int kblocks, double *out, const long long *off_m,
                     const long long *off_n, double alpha, double beta, int ksplit, double *partial, int *status,
                     cudaStream_t st)
{
    const size_t smem = TC_STAGES * TC_STAGE_BYTES + 1024;
    // the attribute is set once per device: launches may be captured into
    // CUDA graphs, and nothing but the launch itself should run per call
    static bool attr_set[KIND_BF16 + 1][64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return check_launch("cudaGetDevice");
    if (!attr_set[KIND][dev]) {
        if (cudaFuncSetAttribute(tc_split_gemm_kernel<KIND>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess)
            return check_launch("cudaFuncSetAttribute(tc_split_gemm_kernel)");
        attr_set[KIND][dev] = true;
    }
    const int mt = (m_pad + TC_BM - 1) / TC_BM, nt = (n_pad + TC_BN - 1) / TC_BN;
    const int per = (kblocks + ksplit - 1) / ksplit;
    const int nsplit = (kblocks + per - 1) / per;           // every split non-empty
    tc_split_gemm_kernel<KIND><<<(unsigned)((long long)mt * nt * nsplit), TC_THREADS, smem, st>>>(
        ma, mal, mb, mbl, M, N, mt, nt, kblocks, per, out, off_m, off_n, alpha, beta, nsplit > 1 ? partial : nullptr,
        status);
    int rc = check_launch("tc_split_gemm_kernel");
    if (rc || nsplit == 1) return rc;
    const long long mn = (long long)M * N;
    const int blocks = (int)std::min<long long>((mn + 255) / 256, 148ll * 16);
    splitk_reduce_kernel<<<blocks, 256, 0, st>>>(partial, nsplit, M, N, out, off_m, off_n, alpha, beta);
    return check_launch("splitk_reduce_kernel");
}

}  // namespace cb

using namespace cb;

extern "C" {

int ccsd_b200_wait_probe(int *status, long long limit_ns, int code, void *stream)
{
    if (!status || limit_ns <= 0 || limit_ns > 10000000000ll || code == 0) {
        set_error("ccsd_b200_wait_probe: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    wait_probe_kernel<<<1, 32, 0, (cudaStream_t)stream>>>(status, (unsigned long long)limit_ns, code);
    return check_launch("wait_probe_kernel");
}

int ccsd_b200_split_pack(int kind, const double *src1, const long long *o1r, const long long *o1k, double c1,
                         const double *src2, const long long *o2r, const long long *o2k, double c2, int rows, int K,
                         int rows_pad, int k_pad, void *hi, void *lo, int rowfast, void *stream)
{
    if ((kind != KIND_TF32 && kind != KIND_BF16) || !src1 || !o1r || !o1k || rows < 0 || K < 0 ||
        rows_pad < rows || k_pad < K || !hi || !lo || (src2 && (!o2r || !o2k)) ||
        k_pad % (16 / (kind == KIND_TF32 ? 4 : 2))) {
        set_error("ccsd_b200_split_pack: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    if ((long long)rows_pad * k_pad == 0) return CCSD_B200_OK;
    const int nrt = (rows_pad + 31) / 32;
    dim3 grid((unsigned)((k_pad + 31) / 32), (unsigned)(nrt < 65535 ? nrt : 65535));
    cudaStream_t st = (cudaStream_t)stream;
#define CB_PACK(KD, RF)                                                                                     \
    split_pack_kernel<KD, RF><<<grid, 256, 0, st>>>(src1, o1r, o1k, c1, src2, o2r, o2k, c2, rows, K, rows_pad, \
                                                    k_pad, hi, lo)
    if (kind == KIND_TF32) {
        if (rowfast) CB_PACK(KIND_TF32, true); else CB_PACK(KIND_TF32, false);
    } else {
        if (rowfast) CB_PACK(KIND_BF16, true); else CB_PACK(KIND_BF16, false);
    }
#undef CB_PACK
    return check_launch("split_pack_kernel");
}

int ccsd_b200_tc_split_gemm(int kind, const void *a_hi, const void *a_lo, const void *b_hi, const void *b_lo, int M,
                            int N, int m_pad, int n_pad, int k_pad, double *out, const long long *off_m,
                            const long long *off_n, double alpha, double beta, int ksplit, double *partial,
                            int *status, void *stream)
{
    const int kstep = TC_ROWB / (kind == KIND_TF32 ? 4 : 2);
    if (ksplit < 1 || (ksplit > 1 && !partial) ||
        (long long)((m_pad + TC_BM - 1) / TC_BM) * ((n_pad + TC_BN - 1) / TC_BN) * ksplit > 2147483647ll) {
        set_error("ccsd_b200_tc_split_gemm: invalid split-K arguments");
        return CCSD_B200_ERR_ARG;
    }
    if ((kind != KIND_TF32 && kind != KIND_BF16) || !a_hi || !a_lo || !b_hi || !b_lo || !out || !off_m || !off_n ||
        !status || M <= 0 || N <= 0 || m_pad < M || n_pad < N || k_pad <= 0 ||
        k_pad % (16 / (kind == KIND_TF32 ? 4 : 2))) {
        set_error("ccsd_b200_tc_split_gemm: invalid argument");
        return CCSD_B200_ERR_ARG;
    }
    CUtensorMap ma, mal, mb, mbl;
    int rc;
    if ((rc = make_map(&ma, a_hi, kind, m_pad, k_pad)) || (rc = make_map(&mal, a_lo, kind, m_pad, k_pad)) ||
        (rc = make_map(&mb, b_hi, kind, n_pad, k_pad)) || (rc = make_map(&mbl, b_lo, kind, n_pad, k_pad)))
        return rc;
    cudaStream_t st = (cudaStream_t)stream;
    const int kblocks = (k_pad + kstep - 1) / kstep;
    if (kind == KIND_TF32)
        return launch_tc<KIND_TF32>(ma, mal, mb, mbl, M, N, m_pad, n_pad, kblocks, out, off_m, off_n, alpha, beta,
                                    ksplit, partial, status, st);
    return launch_tc<KIND_BF16>(ma, mal, mb, mbl, M, N, m_pad, n_pad, kblocks, out, off_m, off_n, alpha, beta,
                                ksplit, partial, status, st);
}

}  // extern "C"
