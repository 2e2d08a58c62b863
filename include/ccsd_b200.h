/*
 * ccsd_b200.h -- C ABI of libccsdb200.so (B200 / sm_100a CCSD gradient hot path).
 *
 * Conventions for every entry point:
 *   - all array arguments are DEVICE pointers owned by the caller;
 *   - work is enqueued on `stream` (a cudaStream_t, NULL = legacy default stream)
 *     and the call returns without synchronising;
 *   - the return value is a status: 0 = CCSD_B200_OK, otherwise one of the
 *     CCSD_B200_ERR_* codes, with a message from ccsd_b200_last_error();
 *   - nothing throws across the ABI; the library is not thread-safe for
 *     concurrent calls from several host threads.
 * Shell data use the libcint/PySCF layout: atm rows of 6 int32
 * [Z, ptr_coord, ...], bas rows of 8 int32 [atom, l, nprim, nctr, kappa,
 * ptr_exp, ptr_coeff, 0], env float64.  ERI entry points take DECONTRACTED
 * shells (nctr == 1; split general contractions first) and l <= 4.
 */
#ifndef CCSD_B200_H
#define CCSD_B200_H
#include <stdint.h>
#ifdef __cplusplus
extern "C" {
#endif

#define CCSD_B200_OK 0
#define CCSD_B200_ERR_ARG 1
#define CCSD_B200_ERR_LAUNCH 2
#define CCSD_B200_ERR_TIMEOUT 3
#define CCSD_B200_ERR_NONFINITE 4
#define CCSD_B200_ERR_UNSUPPORTED 5

/* Message of the last failing call (static storage). */
const char *ccsd_b200_last_error(void);

/*
 * Cartesian s2kl block of (ij|kl) (deriv = 0) or d/dr_1 (ij|kl) (deriv = 1)
 * for i-shells [ish0, ish1), all j-shells and all k >= l shell pairs:
 *   out[comp][i - ao_loc[ish0]][j][k*(k+1)/2 + l],  k >= l,
 * comp = x, y, z for deriv = 1.  Every element of the block is written.
 * ao_loc: Cartesian AO offsets of the nbas decontracted shells (nbas + 1
 * entries); nao = ao_loc[nbas]; lmax = max l over the shells.
 * heavy_quartets (int32 x 4, n_heavy entries) must list exactly the block's
 * quartets (i in [ish0, ish1), any j, k >= l) whose Cartesian block has more
 * than 1000 (deriv = 0) or 500 (deriv = 1) functions: those run on the
 * CTA-cooperative kernel (on a
 * library-owned stream fork/joined with `stream` by events), all others on
 * the warp-per-quartet kernel.
 * Replaces fill_int2e_kernel / fill_int2e_ip1_kernel and the per-i-shell
 * launch loop of _compute_cart
 * (ref: ccsd_gpu/cuda/int2e_module.py:130-463, ccsd_gpu/cuda/int2e_gpu.py:39-108,
 *       ccsd_gpu/cuda/int2e_ip1_module.py:273-667, ccsd_gpu/cuda/int2e_ip1_gpu.py:148-216).
 */
int ccsd_b200_eri_s2kl_cart(int deriv, const int32_t *atm, const int32_t *bas, const double *env,
                            int nbas, const int32_t *ao_loc, int ish0, int ish1, int nao, int lmax,
                            const int32_t *heavy_quartets, long long n_heavy, double *out, void *stream);

/*
 * s2kl block in the SPHERICAL basis, computed in one pass: each shell
 * quartet's Cartesian block is transformed to spherical functions in shared
 * memory by the kernel that computed it, and only the spherical block is
 * written.  Shells with l <= 2 only (lmax > 2: CCSD_B200_ERR_UNSUPPORTED; use
 * ccsd_b200_eri_s2kl_cart and ccsd_b200_cart2sph_s2kl).  Arguments as
 * ccsd_b200_eri_s2kl_cart, plus ao_loc_sph (nbas + 1 spherical AO offsets of
 * the decontracted shells) and c2s_d (the 5 x 6 cart->sph factors of a d
 * shell, row s = spherical function, column = Cartesian function; s and p
 * shells are the identity); nao_sph is the spherical AO count and out is
 * (ncomp, ao_loc_sph[ish1] - ao_loc_sph[ish0], nao_sph, nao_sph (nao_sph + 1) / 2).
 * Replaces compute_int2e_gpu / compute_int2e_ip1_gpu's Cartesian kernel plus
 * the dense nao_cart^2 unpack and cart->sph transform
 * (ref: ccsd_gpu/cuda/int2e_gpu.py:110-215, ccsd_gpu/cuda/int2e_ip1_gpu.py:223-330).
 */
int ccsd_b200_eri_s2kl_sph(int deriv, const int32_t *atm, const int32_t *bas, const double *env, int nbas,
                           const int32_t *ao_loc, const int32_t *ao_loc_sph, const double *c2s_d, int ish0, int ish1,
                           int nao_sph, int lmax, const int32_t *heavy_quartets, long long n_heavy, double *out,
                           void *stream);

/*
 * Integrals of an explicit list of shell quartets (int32 x 4 per quartet,
 * [i, j, k, l]), consumed in-kernel: per quartet and component two checksums
 *   qsum[q][comp][0] = sum_f v_f * (1 + (f mod 8)/8),  qsum[q][comp][1] = sum_f v_f^2
 * over the Cartesian functions f = ((fi*nfj + fj)*nfk + fk)*nfl + fl.
 * Used by the ERI throughput benchmark and its parity checks; no counterpart
 * in the reference (which only stores full blocks, ref: ccsd_gpu/cuda/int2e_gpu.py:81-106).
 */
int ccsd_b200_eri_quartet_checksums(int deriv, const int32_t *atm, const int32_t *bas, const double *env,
                                    const int32_t *quartets, long long nq, int lmax, double *qsum,
                                    void *stream);

/*
 * Heavy-quartet threshold of the list entry points (quartet checksums,
 * ccsd_b200_eri_ip1_contract, ccsd_b200_eri_full_cart) for derivative order
 * deriv (0 or 1): quartets whose Cartesian block has more than nf functions
 * run on the CTA-cooperative kernel, the others one warp each.  Defaults
 * 1000 (int2e) and 500 (int2e_ip1); set by the autotuner (process-wide, all
 * devices).  The get call returns the current value, -1 for a bad deriv.  No
 * counterpart in the reference (its launch shape is fixed,
 * ref: ccsd_gpu/cuda/int2e_ip1_gpu.py:148-216).
 */
int ccsd_b200_eri_set_heavy_nf(int deriv, int nf);
int ccsd_b200_eri_get_heavy_nf(int deriv);

/*
 * Accumulation path of the warp kernels per L-class, for derivative order
 * deriv (0 or 1): choice[c], c = li*27 + lj*9 + lk*3 + ll over the 81
 * classes with every l <= 2 in the quartet's own shell order, is 0 for the
 * compiled rule, 1 for the contracted-HRR path whenever the quartet fits it,
 * 2 for the per-output path; n must be 81.  Applies to the s2kl block entry
 * and the list entry points (process-wide, all devices); set by the
 * autotuner.  The get call writes the current table.  No counterpart in the
 * reference (one code path per kernel, ref: ccsd_gpu/cuda/int2e_ip1_module.py:273-667).
 */
int ccsd_b200_eri_set_paths(int deriv, const uint8_t *choice, int n);
int ccsd_b200_eri_get_paths(int deriv, uint8_t *choice, int n);

/*
 * Cartesian -> spherical transform of an s2kl block:
 * cart (ncomp, nfc, naoc, naoc(naoc+1)/2) -> out (ncomp, nfs, naos, naos(naos+1)/2),
 * tmp (ncomp, nfs, naos, naoc(naoc+1)/2) is caller-provided scratch.  The
 * transform matrix is given by columns in CSR form: spherical function s of
 * the i-block has coefficients val_i[ptr_i[s]..ptr_i[s+1]) on Cartesian rows
 * idx_i[...] of the block; (ptr, idx, val) is the same for the whole basis.
 * Replaces _cart_to_sph_eri0 / _cart_to_sph_eri1, which unpack to a dense
 * nao_cart^2 square (ref: ccsd_gpu/cuda/int2e_gpu.py:115-179,
 * ccsd_gpu/cuda/int2e_ip1_gpu.py:223-289).
 */
int ccsd_b200_cart2sph_s2kl(const double *cart, double *tmp, double *out, int ncomp, int nfc, int naoc,
                            int nfs, int naos, const int32_t *ptr_i, const int32_t *idx_i,
                            const double *val_i, const int32_t *ptr, const int32_t *idx,
                            const double *val, void *stream);

/*
 * ccsd_b200_cart2sph_s2kl without the caller's scratch buffer.  No counterpart
 * in the reference: it exists for callers that cannot allocate device
 * memory -- applications that hand this library a device they already manage
 * with their own pool, or that forbid allocation while a step runs because
 * cudaMalloc can synchronise the device.  The transform's intermediate
 * (ncomp * nfs * naos * naoc(naoc+1)/2 doubles) lives in a fixed 32 MiB device
 * array inside the library, reserved on every GPU that loads it until the
 * process exits.  Larger blocks are rejected with CCSD_B200_ERR_ARG and a
 * message giving both sizes.  The first call on a device looks up the array's
 * address (cudaGetSymbolAddress) and must come before any stream capture.
 * The address is cached per device and belongs to the device's primary
 * context, which is assumed to live for the whole process (do not call this
 * after a cudaDeviceReset).  All calls share the array, so calls that overlap
 * on the GPU race and must be serialised by the caller.  Allocates nothing;
 * arguments and result as in ccsd_b200_cart2sph_s2kl.
 */
int ccsd_b200_cart2sph_s2kl_noalloc(const double *cart, double *out, int ncomp, int nfc, int naoc, int nfs,
                                    int naos, const int32_t *ptr_i, const int32_t *idx_i, const double *val_i,
                                    const int32_t *ptr, const int32_t *idx, const double *val, void *stream);

/*
 * One-electron integrals over DECONTRACTED Cartesian shells, full matrix
 * out[comp][i][j] (nao = ao_loc[nbas]):
 *   op 0 overlap, 1 kinetic, 2 nuclear attraction sum_C -Z_C/|r-C|,
 *   3 1/|r - R_origin| (origin_atom), and 4..7 the same with d/dr on the
 *   first function (3 components x, y, z).
 * Replaces libcint's int1e_ovlp/kin/nuc/rinv and int1e_ipovlp/ipkin/ipnuc/iprinv,
 * which the reference reaches through PySCF's hcore_generator and get_ovlp
 * (ref: ccsd_gpu/gpu_ccsd_grad.py:554-584).
 */
int ccsd_b200_int1e_cart(int op, const int32_t *atm, int natm, const int32_t *bas, int nbas, const double *env,
                         const int32_t *ao_loc, int lmax, int origin_atom, double *out, void *stream);

/*
 * FP64 FMA throughput probe: `blocks` x 256 threads, each running 8
 * independent FMA chains for `iters` iterations (2*8*iters*256*blocks FLOPs).
 * `out` needs blocks*256 doubles (written only in a practically unreachable
 * branch).  Used to measure the FP64 roofline of the ERI kernels; no
 * counterpart in the reference.
 */
int ccsd_b200_fp64_fma_probe(double *out, int blocks, int iters, void *stream);

/*
 * Dense Cartesian ERI tensor from the unique shell quartets: for every
 * quartet (I, J, K, L) of `quartets` (decontracted shells; the caller lists
 * each unique quartet once, e.g. I >= J, K >= L, IJ >= KL) the (IJ|KL) block
 * is computed once and written to all eight index orders of
 * out[nao][nao][nao][nao] (FP64, Cartesian AO order of ao_loc).  Replaces the
 * repeated s2kl blocks (all I, all J) that the reference's SCF/Imat path
 * requests (ref: ccsd_gpu/cuda/int2e_gpu.py:186-215 called per i-shell
 * block, ccsd_gpu/gpu_ccsd_grad.py:436-441) when the whole tensor is needed.
 */
int ccsd_b200_eri_full_cart(const int32_t *atm, const int32_t *bas, const double *env, const int32_t *ao_loc,
                            int nao, const int32_t *quartets, long long nq, int lmax, double *out, void *stream);

/*
 * Two-electron part of the nuclear gradient without storing ERI derivatives:
 * for every shell quartet q = (I, J, K, L) of `quartets` (decontracted shells,
 * K >= L, derivative on I) the (dI J|K L) block is built shell quartet by shell
 * quartet and contracted at once with the density `gamma`,
 *   qwork[q][x] = w_q * sum_{ijkl in q} (d/dx_i ij|kl) gamma[i][j][k][l],
 * w_q = 1 if K == L else 2 (gamma must be symmetric in k <-> l; dense
 * [nao]^4, FP64, in the Cartesian AO basis of ao_loc).  Then
 *   out[s][x] = sum_{q in [seg[s], seg[s+1])} qwork[q][x]
 * in a fixed order (list sorted by the atom of I gives per-atom gradients).
 * qwork holds nq * 3 doubles, out nseg * 3.  Replaces the int2e_ip1 -> Gamma
 * contraction loop of the Phase-3 gradient, which stores the derivative
 * integrals of each atom block (ref: ccsd_gpu/gpu_ccsd_grad.py:416-500,
 * ccsd_gpu/cuda/int2e_ip1_gpu.py:148-330).
 */
int ccsd_b200_eri_ip1_contract(const int32_t *atm, const int32_t *bas, const double *env, const int32_t *ao_loc,
                               int nao, const double *gamma, const int32_t *quartets, long long nq,
                               const long long *seg, int nseg, int lmax, double *qwork, double *out, void *stream);

/*
 * The same contraction with only rows [row0, row0 + nrows) of gamma held:
 * gamma_rows is (nrows, nao, nao, nao), row r holding gamma[row0 + r].  Meant
 * for one atom's segment of the quartet list (every I-shell function of the
 * quartets inside the rows), so the gradient of a large molecule is streamed
 * atom block by atom block and never holds the whole [nao]^4 density, as the
 * reference streams its gradient loop by shell blocks sized from max_memory
 * (ref: ccsd_gpu/gpu_ccsd_grad.py:416-432).  Functions outside the rows
 * contribute zero (a bounds guard, not an error).
 */
int ccsd_b200_eri_ip1_contract_rows(const int32_t *atm, const int32_t *bas, const double *env,
                                    const int32_t *ao_loc, int nao, const double *gamma_rows, int row0, int nrows,
                                    const int32_t *quartets, long long nq, const long long *seg, int nseg, int lmax,
                                    double *qwork, double *out, void *stream);

/*
 * Failure-path probe (no counterpart in the reference): one thread waits,
 * with the same bounded mbarrier wait the tensor-core GEMM pipeline uses, on
 * a barrier that nothing arrives at.  After limit_ns (<= 10 s) of global
 * timer the wait gives up, `code` is stored in *status (if it was 0) and the
 * kernel returns normally, so the host reads the error and the context stays
 * usable.  Used by the tests of the timeout path.
 */
int ccsd_b200_wait_probe(int *status, long long limit_ns, int code, void *stream);

/*
 * Split-precision tensor-core contraction, step 1: gather + split.
 *   v[r][k] = c1 * src1[o1r[r] + o1k[k]] + c2 * src2[o2r[r] + o2k[k]]   (src2 may be NULL)
 * for r < rows, k < K (zero elsewhere), written as hi + lo parts, K-major,
 * [rows_pad x k_pad]: kind 0 = TF32 (float storage, 4 B), kind 1 = BF16 (2 B).
 * rows_pad >= rows; k_pad >= K and a multiple of 4 (TF32) / 8 (BF16), so
 * that every row starts on a 16-byte boundary.  No padding to the 128-row
 * GEMM tile is needed: the GEMM's TMA loads read zeros past the array.
 * rowfast != 0 tells that src1 is contiguous along the packed rows (a
 * transposing gather): the kernel then reads along rows and turns 32 x 32
 * tiles through shared memory, so reads and writes are both coalesced.
 * The offset tables (int64, element units) express any strided or permuted
 * view of the FP64 operands.  Replaces the operand transposes/copies that
 * precede the CuPy einsum contractions of the Lambda and RDM builders
 * (ref: ccsd_gpu/gpu_ccsd_lambda.py:68-337, ccsd_gpu/gpu_ccsd_grad.py:101-246).
 */
int ccsd_b200_split_pack(int kind, const double *src1, const long long *o1r, const long long *o1k, double c1,
                         const double *src2, const long long *o2r, const long long *o2k, double c2, int rows,
                         int K, int rows_pad, int k_pad, void *hi, void *lo, int rowfast, void *stream);

/*
 * Split-precision tensor-core contraction, step 2 (tcgen05 + TMA + TMEM):
 *   out[off_m[m] + off_n[n]] = alpha * sum_k (Ahi Bhi + Ahi Blo + Alo Bhi)[m,n,k] + beta * out[...]
 * for m < M, n < N.  The tensor cores accumulate in FP32 over chunks of
 * 512 k; each chunk is added to the output in FP64.  Operands come from
 * ccsd_b200_split_pack (A: [m_pad x k_pad], B: [n_pad x k_pad], m_pad >= M,
 * n_pad >= N, k_pad a multiple of 4 (TF32) / 8 (BF16)).  Split-K: with ksplit > 1 the k blocks are
 * divided over up to ksplit CTAs per output tile; each writes an FP64
 * partial tile into `partial` (caller-allocated, ksplit * M * N doubles) and a
 * second kernel sums the partials in a fixed order and applies alpha/beta, so
 * results do not depend on scheduling.  ksplit = 1 needs no `partial`.
 * `status` (one int, zero-initialised by the
 * caller) receives a non-zero code if a pipeline wait expired.  Replaces the
 * cuTENSOR/cuBLAS einsum contractions of the Lambda solver and density
 * builders, and the CPU vvvv ladder term (ref: ccsd_gpu/gpu_ccsd_lambda.py:238-241).
 */
int ccsd_b200_tc_split_gemm(int kind, const void *a_hi, const void *a_lo, const void *b_hi, const void *b_lo,
                            int M, int N, int m_pad, int n_pad, int k_pad, double *out, const long long *off_m,
                            const long long *off_n, double alpha, double beta, int ksplit, double *partial,
                            int *status, void *stream);

#ifdef __cplusplus
}
#endif
#endif
