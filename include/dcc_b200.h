/*
 * dcc_b200.h -- C ABI of the B200 (sm_100a) library for Distributed-CC's
 * triples/quadruples hot path.
 *
 * Conventions
 *  - Tensor arguments are DEVICE pointers to C-contiguous float64 (or the
 *    stated integer type) buffers owned by the caller; the library writes in
 *    place exactly like the reference helpers and allocates nothing unless an
 *    entry point says so.  Arguments documented as "host" are host pointers.
 *  - `stream` is a cudaStream_t passed as void*; NULL is the legacy stream.
 *    Calls are asynchronous on that stream unless documented otherwise.
 *  - Every entry point returns DCC_OK (0) or an error code; dcc_last_error()
 *    then holds a message for the calling thread.  Nothing aborts.
 *  - Pattern names are the reference's strings ("P3_full", "P4_444", ...).
 *
 * Each declaration names the reference interface it replaces, by file:line in
 * the Distributed-CC project (the reference binds those through ctypes in
 * distr_cc/_c_rccsdt.py, distr_cc/_c_rccsdt_q.py, distr_cc/_c_rccsdtq.py).
 */
#ifndef DCC_B200_H
#define DCC_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define DCC_API __attribute__((visibility("default")))
#else
#define DCC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

enum {
    DCC_OK = 0,
    DCC_ERR_PATTERN = 1,     /* unknown pattern string */
    DCC_ERR_SHAPE = 2,       /* inconsistent sizes / indices out of range */
    DCC_ERR_NULL = 3,        /* required pointer is NULL */
    DCC_ERR_CUDA = 4,        /* CUDA runtime / launch failure */
    DCC_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
    DCC_ERR_UNSUPPORTED = 6, /* valid request the library does not implement */
    DCC_ERR_NOT_LOCAL = 7,   /* requested block is not stored (reference: silent no-op) */
    DCC_ERR_WORKSPACE = 8    /* workspace argument too small */
};

/* Message for the last failing call on this thread ("" after success). */
DCC_API const char *dcc_last_error(void);
/* Library ABI version (major*100 + minor). */
DCC_API int dcc_version(void);

/* ----------------------------------------------------------------------
 * T3 helpers (replace src/rccsdt.c)
 * ---------------------------------------------------------------------- */

/* A <- beta*A + alpha*P(A) on one nvir^3 block; P = P3_full | P3_422 | P3_201.
 * Replaces t3_single_spin_summation_inplace_ (src/rccsdt.c:131-233). */
DCC_API int dcc_t3_single_spin_summation_inplace(double *A, int64_t nvir, const char *pattern, double alpha,
                                         double beta, void *stream);

/* Same on nblocks consecutive nvir^3 blocks in one launch.  Replaces the
 * multi-block t3_spin_summation_inplace_(r3, n3, nvir, "P3_full", -1/6, 1)
 * called at distr_cc/rccsdt.py:947 (PySCF pyscf/cc/rccsdt.py). */
DCC_API int dcc_t3_spin_summation_inplace(double *A, int64_t nblocks, int64_t nvir, const char *pattern, double alpha,
                                  double beta, void *stream);

/* U[o] = the canonical T3 (t3, [n3][nvir]^3, i<=j<=k blocks in lexicographic order) unpacked to
 * every ordered (i,j,k) o (U: [nocc^3][nvir]^3, o = (i*nocc+j)*nocc+k, as dcc_t3_unpack_all) and
 * X[o] = beta*U[o] + alpha*P(U[o]) (the P3 pattern of dcc_t3_spin_summation, bit-identical to it
 * applied to U), in one pass over the canonical blocks; U may be NULL (X alone).  The
 * take_t3_single_local + t3_single_spin_summation_inplace_(.., "P3_201") of every ordering that
 * r1r2_add_t3_tri_ / intermediates_t3_add_t3_tri make per block (distr_cc/rccsdt.py:308-309,
 * 351-352), for all blocks at once.  t3, U and X must not overlap. */
DCC_API int dcc_t3_unpack_p3(const double *t3, double *U, double *X, int64_t nocc, int64_t nvir, const char *pattern,
                             double alpha, double beta, void *stream);

/* B = beta*A + alpha*P(A) block by block, out of place (A and B do not overlap, or
 * B == A for the in-place form above); same patterns and arithmetic.  The
 * out-of-place t3_spin_summation of PySCF's rccsdt_highm as the reference calls it
 * (distr_cc/rccsdtq.py:853, P3_201 of the full T3 with alpha 1, beta 0). */
DCC_API int dcc_t3_spin_summation(const double *A, double *B, int64_t nblocks, int64_t nvir, const char *pattern,
                                  double alpha, double beta, void *stream);

/* Diagnostic: dcc_t3_spin_summation through one chosen kernel: 0 the default choice, 1 strips
 * (the patterns with p4 = 0, i.e. P3_201, at nvir <= 104), 2 orbit tiles (every pattern).
 * DCC_ERR_UNSUPPORTED (nothing launched) where the kernel does not apply.  Same results. */
/* B = beta*A + alpha*P(A) out of place on FP32 blocks (the arithmetic in FP64 on the FP32
 * values, the result rounded once): X = P3_201 of the FP32 unpacked T3 that the split-precision
 * feedback strings read (distr_cc/rccsdt.py:308-309, 351-352).  The patterns without a p4 term,
 * nvir <= 104. */
DCC_API int dcc_t3_spin_summation_f32(const float *A, float *B, int64_t nblocks, int64_t nvir, const char *pattern,
                                      double alpha, double beta, void *stream);

DCC_API int dcc_t3_spin_summation_kernel(const double *A, double *B, int64_t nblocks, int64_t nvir,
                                         const char *pattern, double alpha, double beta, int kernel, void *stream);

/* B0 = 2T - T_acb - T_cba, B1 = 2T - T_bac - T_acb, B2 = B0 + T_acb - T_bac on
 * nblocks blocks.  Replaces t3_spin_summation_triple_sym_ (src/rccsdt.c:245-310). */
DCC_API int dcc_t3_spin_summation_triple_sym(const double *A, double *B0, double *B1, double *B2, int64_t nblocks,
                                     int64_t nvir, void *stream);

/* B[a,b,c] = A[a,b,c] + A[c,a,b] on nblocks blocks.
 * Replaces t3_transpose_add_ (src/rccsdt.c:320-375). */
DCC_API int dcc_t3_transpose_add(const double *A, double *B, int64_t nblocks, int64_t nvir, void *stream);

/* Diagnostic: moves every orbit tile set of nblocks nvir^3 blocks through the
 * spin-summation kernel's TMA loads and stores with no arithmetic (A is left
 * unchanged): the traffic ceiling of that kernel on this layout.  Even nvir
 * and a 16-byte aligned A only (else DCC_ERR_UNSUPPORTED).  No reference
 * counterpart. */
DCC_API int dcc_t3_orbit_roundtrip(double *A, int64_t nblocks, int64_t nvir, void *stream);

/* Copies into *out (host int) the status word of the bounded waits of the
 * TMA spin-summation kernel on the current device (0, or DCC_ERR_TIMEOUT
 * once a wait gave up) and clears it; synchronizes `stream`.  No reference
 * counterpart: the reference symmetrizers run on the host. */
DCC_API int dcc_t3_symmetrize_status(int *out, void *stream);

/* t3_blk = T3[i,j,k] for any ordering, unpacked from canonical storage.
 * ijk_to_local_idx is a HOST array of nocc3 int64 (-1: not stored).  Returns
 * DCC_ERR_NOT_LOCAL when the block is not stored (the reference silently
 * returns).  Replaces take_t3_ijk_single_ (src/rccsdt.c:119-129). */
DCC_API int dcc_take_t3_ijk_single(const double *t3_local, double *t3_blk, const int64_t *ijk_to_local_idx, int64_t i,
                           int64_t j, int64_t k, int64_t nocc, int64_t nvir, void *stream);

/* Batched unpack: out[n] = T3[ijk[n][0], ijk[n][1], ijk[n][2]] for n < count;
 * ijk (int32 [count][3]) and ijk_to_local_idx (int64 [nocc3]) are DEVICE
 * arrays.  Blocks that are not stored are zero-filled.  Batched form of
 * take_t3_ijk_single_ (src/rccsdt.c:119-129) as used by
 * distr_cc/rccsdt.py:266-267,300. */
DCC_API int dcc_take_t3_batched(const double *t3_local, double *out, const int32_t *ijk, const int64_t *ijk_to_local_idx,
                        int64_t count, int64_t nocc, int64_t nvir, void *stream);

/* U[(x*nocc + y)*nocc + z] = T3[x,y,z] for every ordered occupied triple (U is
 * DEVICE [nocc^3][nvir^3]) from the canonical blocks of one rank: the
 * all-orderings form of take_t3_ijk_single_ (src/rccsdt.c:119-129), reading
 * every canonical block once. */
DCC_API int dcc_t3_unpack_all(const double *t3, double *U, int64_t nocc, int64_t nvir, void *stream);

/* The same into an FP32 U (each value rounded once), the copy of T3 that the split-precision
 * contractions read (their bf16 / tf32 pieces keep fewer bits than FP32); nvir <= 104. */
DCC_API int dcc_t3_unpack_all_f32(const double *t3, float *U, int64_t nocc, int64_t nvir, void *stream);

/* send_data[r] = t3_local[ijk_to_local_idx[requests[r]]] for stored blocks
 * (DEVICE index arrays).  Replaces fill_local_data_ijk_ (src/rccsdt.c:105-117). */
DCC_API int dcc_fill_local_data_ijk(const double *t3_local, double *send_data, const int32_t *requests,
                            const int64_t *ijk_to_local_idx, int64_t n_requests, int64_t nvir, void *stream);

/* r3[q,a,b,c] /= eia[i,a] + eia[j,b] + eia[k,c] for the canonical triple
 * (i,j,k) = ijk[q] (DEVICE int32 [nblocks][3]; eia DEVICE [nocc][nvir],
 * already including -level_shift).  Replaces r3_tri_divide_e_
 * (distr_cc/rccsdt.py:734-744). */
DCC_API int dcc_r3_tri_divide_e(double *r3, const double *eia, const int32_t *ijk, int64_t nblocks, int64_t nvir,
                        void *stream);

/* Fused T3 update: r3 /= D (as dcc_r3_tri_divide_e), t3 += r3, and
 * norms[0] = sum r3^2, norms[1] = sum over a,b,c < nvir_active of r3^2
 * (DEVICE double[2]).  write_r3 != 0 also stores the divided r3.  The
 * workspace (DEVICE, >= dcc_t3_update_workspace_bytes()) holds per-CTA
 * partial sums.  Replaces distr_cc/rccsdt.py:949-971. */
DCC_API size_t dcc_t3_update_workspace_bytes(int64_t nblocks, int64_t nvir);
DCC_API int dcc_t3_divide_update(double *t3, double *r3, const double *eia, const int32_t *ijk, int64_t nblocks,
                         int64_t nvir, int64_t nvir_active, int write_r3, double *norms, void *workspace,
                         size_t workspace_bytes, void *stream);

/* The same fused update for callers that cannot allocate device memory: a
 * host runtime that owns every device allocation through its own pool and
 * forbids libraries to call cudaMalloc, or a thin ctypes caller (like the
 * reference's wrappers) that holds only the amplitude tensors and has no
 * allocator to obtain a workspace from.  No counterpart in the reference
 * (its C helpers run on the host and malloc their scratch).
 * The per-CTA partial sums live in a static 128 KiB device array inside the
 * library (every GPU that loads the library holds it until exit), so this
 * call allocates nothing; it serves nblocks * nvir^2 <= 8 388 608 rows and
 * returns DCC_ERR_SHAPE with a message beyond that.  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress); make
 * that first call before any stream capture.  All calls on a device share
 * the array, so calls that overlap on the GPU (different streams, no
 * ordering between them) race on it. */
DCC_API int dcc_t3_divide_update_noalloc(double *t3, double *r3, const double *eia, const int32_t *ijk,
                                         int64_t nblocks, int64_t nvir, int64_t nvir_active, int write_r3,
                                         double *norms, void *stream);

/* IJK -> ABC layout transform at one rank: t3_abc[g][x][y][z] (g the rank of
 * a<=b<=c) from t3_ijk[q][a][b][c] (q the rank of i<=j<=k).  Reproduces the
 * record pack + Alltoallv + unpack of distr_cc/distribute_t3.py:1544-1642 with
 * src/rccsdt.c:411-561 (last record wins where records collide). */
DCC_API int dcc_redistribute_ijk_to_abc(const double *t3_ijk, double *t3_abc, int64_t nocc, int64_t nvir, void *stream);

/* target[ia][ib][c][i][j][k] (row pitch ld_b over ib) for a in [a0,a1),
 * b in [b0,b1), all c, from ABC storage t3_abc[g][x][y][z] with the occupied
 * axes permuted by the virtual ordering case.  Replaces fill_t3_from_ptr_array
 * (src/rccsdt_q.c:655-828); at one rank every ABC block is local, so the
 * pointer table becomes one contiguous array. */
DCC_API int dcc_fill_t3_from_abc(double *target, int64_t a0, int64_t a1, int64_t b0, int64_t b1, int64_t nvir,
                         int64_t nocc, const double *t3_abc, int64_t ld_b, void *stream);

/* r3[q][a][b][c] = beta*r3 + sum_s scale_s * sum_sigma U_s(sigma(i,j,k), sigma(a,b,c))
 * over the six simultaneous permutations sigma of (i,j,k) and (a,b,c), for the
 * canonical triples ijk[q] (DEVICE int32 [nblocks][3]).  U_s is addressed by
 * HOST strides {x,y,z,a,b,c} (in doubles); the second source is optional
 * (u1 == NULL).  Replaces the twelve per-block einsums W_vvvo.t2 / W_vooo.t2
 * of compute_r3_tri (distr_cc/rccsdt.py:385-396): each group of six is the
 * S3 symmetrization of one contraction over all ordered (i,j,k). */
DCC_API int dcc_t3_s3_gather(double *r3, const int32_t *ijk, int64_t nblocks, int64_t nvir, double beta,
                             const double *u0, double scale0, const int64_t *strides0, const double *u1,
                             double scale1, const int64_t *strides1, void *stream);

/* General form: r3[q][abc] = beta*r3 + sum_s scales[s] * sum_{p in masks[s]} U_s(p(ijk), p(abc))
 * for nsrc <= 4 sources (HOST arrays: bases[s], scales[s], strides[6*s..6*s+5],
 * masks[s] = 6-bit subset of the simultaneous permutations in the order
 * (x,y,z), (x,z,y), (y,x,z), (y,z,x), (z,x,y), (z,y,x)); at most 12 (source,
 * permutation) pairs.  Used for the W.t2 terms and the OO batch terms of
 * compute_r3_tri (distr_cc/rccsdt.py:385-396, 435-732). */
DCC_API int dcc_t3_perm_gather(double *r3, const int32_t *ijk, int64_t nblocks, int64_t nvir, double beta, int nsrc,
                               const double *const *bases, const double *scales, const int64_t *strides,
                               const int *masks, void *stream);

/* dcc_t3_perm_gather for sources laid out as blocks of nocc-digit (x, y, z)
 * (nocc is needed for the block coordinates): one persistent kernel in which
 * a producer warp moves each (source, permutation) tile with a TMA box load
 * and the summed tile leaves through a TMA store.  Falls back to the
 * cp.async kernel when a source does not fit the copy engine (odd nvir, a
 * non-unit c stride, b slower than a, or block strides that do not collapse
 * into two dimensions).  *status (DEVICE int, zero before the call) becomes
 * DCC_ERR_TIMEOUT if a bounded wait gave up. */
DCC_API int dcc_t3_perm_gather_tma(double *r3, const int32_t *ijk, int64_t nblocks, int64_t nocc, int64_t nvir,
                                   double beta, int nsrc, const double *const *bases, const double *scales,
                                   const int64_t *strides, const int *masks, int *status, void *stream);
/* The S3 gather of compute_r3_tri's terms (distr_cc/rccsdt.py:385-396, 435-732, as the sum over
 * the six simultaneous permutations of one full-layout tensor) from an FP32 S [nocc^3][nvir^3]:
 *   r3[q][a,b,c] = beta r3 + scale sum_p S[p(ijk_q)][p(abc)],
 * summed in FP64 in the order of dcc_t3_perm_gather_tma.  S is the split precisions' FP32
 * accumulator of the residual's GEMMs (dcc_gemm_split3_ld4_f32c); nvir <= 104. */
DCC_API int dcc_t3_s3_gather_f32(double *r3, const int32_t *ijk, int64_t nblocks, int64_t nocc, int64_t nvir,
                                 double beta, const float *S, double scale, void *stream);

/* ----------------------------------------------------------------------
 * Device DIIS (replaces the vector passes of distr_cc/diis.py:105-177 as
 * driven by run_diis_t3, distr_cc/rccsdt.py:1026-1067)
 * ---------------------------------------------------------------------- */

/* Bytes of the workspace both DIIS passes take (per-CTA partial sums). */
DCC_API size_t dcc_diis_workspace_bytes(void);

/* Length of the DIIS vector (xprev and every slot) for nseg <= 4 segments of seg_n[s]
 * doubles: segment s occupies [seg_off[s], seg_off[s] + seg_n[s]) (seg_off, HOST, may be
 * NULL), every segment starting on a multiple of 32 elements; the gaps are zero.  -1 on
 * bad sizes.  The vector of DIIS.update (distr_cc/diis.py:105-177) in this layout. */
DCC_API int64_t dcc_diis_vector_length(const int64_t *seg_n, int nseg, int64_t *seg_off);

/* v = concat(seg_scale[s] * seg[s]) (nseg <= 4 DEVICE segments of seg_n[s]
 * doubles, HOST tables, laid out as dcc_diis_vector_length gives; xprev and the
 * slots 16-byte aligned); e = v - xprev; x_slot = v; e_slot = e;
 * dots[s] = <e, e_other[s]> for s < nother (<= 15), dots[nother] = <e, e>
 * (DEVICE).  The B-matrix row of DIIS.update (distr_cc/diis.py:121-133). */
DCC_API int dcc_diis_push(double *const *seg, const int64_t *seg_n, const double *seg_scale, int nseg, double *xprev,
                          double *x_slot, double *e_slot, const double *const *e_other, int nother, double *dots,
                          void *workspace, size_t workspace_bytes, void *stream);

/* xnew = sum_s coef[s] xs[s] (HOST coefficients, nd <= 16 DEVICE slots, each
 * product rounded before its addition as distr_cc/diis.py:172-176);
 * delta[0] = |xnew - xprev|^2 (distr_cc/_runtime.py:90); xprev = xnew;
 * out_seg[s] = xnew / seg_scale[s] over the segments (the unpack of
 * distr_cc/_runtime.py:168-187). */
DCC_API int dcc_diis_combine(const double *const *xs, const double *coef, int nd, double *xprev,
                             double *const *out_seg, const int64_t *seg_n, const double *seg_scale, int nseg,
                             double *delta, void *workspace, size_t workspace_bytes, void *stream);

/* ----------------------------------------------------------------------
 * T4 helpers (replace src/rccsdtq.c and PySCF libccsdt.t4_add_)
 * ---------------------------------------------------------------------- */

/* A <- beta*A + alpha*Q(A), Q = 1 - P[4] - P[3,1] on nocc4 blocks of nvir^4.
 * Replaces t4_project_1_minus_p4_p31_inplace_ (src/rccsdtq.c:262-308). */
DCC_API int dcc_t4_project_1_minus_p4_p31_inplace(double *A, int64_t nocc4, int64_t nvir, double alpha, double beta,
                                          void *stream);

/* A <- alpha*P(A) + beta*A on nouter blocks of ninner^4, P = P4_full | P4_444 |
 * P4_442 | P4_201.  Replaces t4_spin_summation_inplace_ (src/rccsdt_q.c:33-472,
 * used with outer = abcd, inner = nocc at distr_cc/rccsdt_q.py:1133) and, with
 * nouter = 1, t4_single_spin_summation_inplace_ (src/rccsdtq.c:316-916). */
DCC_API int dcc_t4_spin_summation_inplace(double *A, int64_t nouter, int64_t ninner, const char *pattern, double alpha,
                                  double beta, void *stream);

/* dst = src + src[c,a,b,d] + src[d,a,c,b].  Replaces t4_transpose_add_
 * (src/rccsdtq.c:990-1005). */
DCC_API int dcc_t4_transpose_add(const double *src, double *dst, int64_t nvir, void *stream);

/* Four P4_201 variants B0..B3.  Replaces t4_spin_summation_quadruple_sym_
 * (src/rccsdtq.c:1018-1047). */
DCC_API int dcc_t4_spin_summation_quadruple_sym(const double *src, double *B0, double *B1, double *B2, double *B3,
                                        int64_t nvir, void *stream);

/* The two above on nblocks consecutive nvir^4 blocks in one launch (nblocks < 65536): the
 * per-source-block forms the OO batch of compute_r4_tri takes (distr_cc/rccsdtq.py:1166-1169,
 * there one block at a time). */
DCC_API int dcc_t4_transpose_add_batched(const double *src, double *dst, int64_t nblocks, int64_t nvir, void *stream);
DCC_API int dcc_t4_spin_summation_quadruple_sym_batched(const double *src, double *B0, double *B1, double *B2,
                                                        double *B3, int64_t nblocks, int64_t nvir, void *stream);

/* The per-block strings of compute_r4_tri (distr_cc/rccsdtq.py:862-1055, the reference's loop
 * over its stored blocks) in ONE launch, FP64:
 *   r4[q][a,b,c,d] = beta r4[q][a,b,c,d] + sum_s alpha_s sum_{k0,k1} W_s[..] T_s[..]
 * for every stored block q (occupied indices quads[q][0..3], DEVICE int32 [nq][4]) and every
 * string s of the DEVICE descriptor table desc[nstr][DCC_T4S_DESC_LEN] (int64):
 *    0 W operand index   1 T operand index      (into ops / op_numel, HOST arrays of nops <= 16)
 *    2-5  W strides of the occupied letters i, j, k, l     6-9  T strides of i, j, k, l
 *   10 W stride of the block index q                      11 T stride of q
 *   12-15 W strides of the output letters a, b, c, d      16-19 T strides of a, b, c, d
 *   20 bit x set: output letter x is in W (its T stride must be 0), else in T (W stride 0)
 *   21 K0  22 W stride  23 T stride of the first summed letter
 *   24 K1  25 W stride  26 T stride of the second (K1 = 1 when there is none)
 *   27 alpha as the bits of an IEEE double
 *   28 row order: nibble p (p = 0 slowest) holds 1 + the output letter at position p of the
 *      rows (the letters of W, each once; 0 = empty position); 29 the same for the columns
 *      (the letters of T); the kernel iterates the last filled position fastest
 *   30 pair mode: the W stride of the pair's occupied index m
 *   31 mode: 0 = a string of the block itself; g + 1 = pair mode for group g < ngroups: the
 *      string runs once for every pair (src, m) = pair_sm[p][0..1] (DEVICE int32 [npairs][2])
 *      with p in [pair_off[q][g], pair_off[q][g+1]) (DEVICE int32 [nq][ngroups+1]); field 11
 *      then strides the source block src instead of q, and W's base moves by m x field 30
 *      (the OO batch's W_ovov / W_voov terms, distr_cc/rccsdtq.py:1062-1349, sparse: only the
 *      (source, output) pairs that exist)
 * An element of an operand is ops[n][sum of stride x index]; strides are in elements.  Every
 * string is bounds-checked against op_numel before it runs; a failing string is skipped and
 * sets bit 2 of *status (DEVICE int), an out-of-range occupied index bit 1, a failing pair
 * bit 4.  ngroups = 0 allows NULL pair lists.  r4 is [nq][nvir^4]; nvir^3 doubles must fit
 * the per-CTA accumulator (nvir <= 29); at most 32 operands, each below 2^31 elements. */
#define DCC_T4S_DESC_LEN 32
DCC_API int dcc_t4_strings(const double *const *ops, const int64_t *op_numel, int nops, const int64_t *desc, int nstr,
                           const int32_t *quads, int64_t nq, const int32_t *pair_off, const int32_t *pair_sm,
                           int ngroups, int64_t npairs, int64_t nocc, int64_t nvir, double beta, double *r4,
                           int *status, void *stream);
/* Output rows a per CTA that dcc_t4_strings uses for nq blocks (-1: nvir too large). */
DCC_API int dcc_t4_strings_rows_per_cta(int64_t nq, int64_t nvir);

/* r4[q] /= eia[i,a]+eia[j,b]+eia[k,c]+eia[l,d] for ijkl = local_ijkl[q]
 * (DEVICE int32 [nlocal][4]).  Replaces r4_local_tri_divide_e_
 * (src/rccsdtq.c:1055-1088). */
DCC_API int dcc_r4_local_tri_divide_e(double *r4_local, const double *eia, const int32_t *local_ijkl, int64_t nlocal,
                              int64_t nvir, void *stream);

/* t4_blk = T4[i,j,k,l] for any ordering; zero-rule blocks are zero-filled.
 * ijkl_to_local_idx is a HOST array over the full triangular index.
 * Replaces unpack_t4_ijkl_single_ (src/rccsdtq.c:1104-1125). */
DCC_API int dcc_unpack_t4_ijkl_single(const double *t4_local, double *t4_blk, const int64_t *ijkl_to_local_idx, int64_t i,
                              int64_t j, int64_t k, int64_t l, int64_t nocc, int64_t nvir, void *stream);

/* send_data[r] = t4_local[ijkl_to_local_idx[requests[r]]] (DEVICE index
 * arrays).  Replaces fill_local_data_ijkl_ (src/rccsdtq.c:1090-1102). */
DCC_API int dcc_fill_local_data_ijkl(const double *t4_local, double *send_data, const int32_t *requests,
                             const int64_t *ijkl_to_local_idx, int64_t n_requests, int64_t nvir, void *stream);

/* t4 += r4 over n doubles.  Replaces PySCF libccsdt t4_add_ as bound at
 * distr_cc/_rccsdtq_core.py:43-48 (elementwise add over nocc4*nvir^4). */
DCC_API int dcc_t4_add(double *t4, const double *r4, int64_t n, void *stream);

/* ----------------------------------------------------------------------
 * (Q) denominator-and-energy loop (replace src/rccsdt_q.c, distr_cc/rccsdt_q.py)
 * ---------------------------------------------------------------------- */

/* r4[abcd][ijkl] /= D, zero where |D| <= 1e-15.  e_occ/e_vir DEVICE.
 * Replaces e_abcdijkl_division_ (src/rccsdt_q.c:474-588). */
DCC_API int dcc_e_abcdijkl_division(double *r4, const double *e_occ, const double *e_vir, int64_t a0, int64_t a1,
                            int64_t b0, int64_t b1, int64_t c0, int64_t c1, int64_t d0, int64_t d1, int64_t blk_a,
                            int64_t blk_b, int64_t blk_c, int64_t blk_d, int64_t nocc, void *stream);

/* t4[abcd][:] *= factor[abcd] (exact zero where factor == 0); factor DEVICE.
 * Replaces t4_multiply_factor_ (src/rccsdt_q.c:590-650). */
DCC_API int dcc_t4_multiply_factor(double *t4_blk, const double *factor_blk, int64_t blk_a, int64_t blk_b, int64_t blk_c,
                           int64_t blk_d, int64_t nocc, void *stream);

/* Fused per-task epilogue of the (Q) loop (distr_cc/rccsdt_q.py:1131-1154):
 *   t~4 = factor(abcd) * P4_444_ijkl((t4 + z4) / D)
 *   out[0] += <t~4, z4sq>/12            ([Q] bracket)
 *   out[1] += <t~4, z4>/12 + that term  ((Q) paren)
 * where z4sq is the disconnected vvoo x t2 product of distr_cc/rccsdt_q.py:1143-1150
 * formed on the fly from eris_vvoo [nvir][nvir][nocc][nocc] and t2_vvoo
 * [nvir][nvir][nocc][nocc] (DEVICE).  t4 and z4 ([blk]^4 x nocc^4, DEVICE) are
 * only read.  out is DEVICE double[2] and is accumulated into.  The workspace
 * (>= dcc_q_epilogue_workspace_bytes()) holds per-CTA partial sums. */
DCC_API size_t dcc_q_epilogue_workspace_bytes(int64_t blksize, int64_t nocc);
DCC_API int dcc_q_task_epilogue(const double *t4, const double *z4, const double *eris_vvoo, const double *t2_vvoo,
                        const double *e_occ, const double *e_vir, int64_t a0, int64_t a1, int64_t b0, int64_t b1,
                        int64_t c0, int64_t c1, int64_t d0, int64_t d1, int64_t blksize, int64_t nocc,
                        int64_t nvir, double *out, void *workspace, size_t workspace_bytes, void *stream);

/* The same epilogue over a whole task group (the tasks sharing a-, b- and
 * c-blocks, d over [d0, d1)): t4 and z4 (DEVICE, float64, or float32 when
 * f32 = 1) are stored [i][j][k][l][a][b][c][d] over the ranges [a0, a1) x
 * [b0, b1) x [c0, c1) x [d0, d1); vvooT and t2T are eris_vvoo and t2_vvoo
 * with the second virtual index fastest, [nvir][nocc][nocc][nvir] (DEVICE).
 * Each (a, b, c, d) of the group enters with its factor (distr_cc/rccsdt_q.py:
 * 410-428), so the sums equal those of the group's tasks.  workspace >=
 * dcc_q_group_epilogue_workspace_bytes(). */
/* Adjoint of dcc_q_group_epilogue (float64 blocks) for the cotangents g_bracket,
 * g_paren of the two energies: writes, for every position of the group block,
 * the gradients of g_bracket [Q] + g_paren (Q) with respect to t4, z4 and the
 * disconnected z4sq (same [i][j][k][l][a][b][c][d] layout, DEVICE).  No
 * counterpart in the reference, which has no (Q) gradient; it is the first
 * step of the hand-written (Q) VJP. */
DCC_API int dcc_q_group_epilogue_adjoint(const double *t4, const double *z4, const double *vvooT, const double *t2T,
                                         const double *e_occ, const double *e_vir, int64_t a0, int64_t a1,
                                         int64_t b0, int64_t b1, int64_t c0, int64_t c1, int64_t d0, int64_t d1,
                                         int64_t nocc, int64_t nvir, double g_bracket, double g_paren, double *gt4,
                                         double *gz4, double *gz4sq, void *stream);
DCC_API size_t dcc_q_group_epilogue_workspace_bytes(void);
DCC_API int dcc_q_group_epilogue(const void *t4, const void *z4, int f32, const double *vvooT, const double *t2T,
                                 const double *e_occ, const double *e_vir, int64_t a0, int64_t a1, int64_t b0,
                                 int64_t b1, int64_t c0, int64_t c1, int64_t d0, int64_t d1, int64_t nocc,
                                 int64_t nvir, double *out, void *workspace, size_t workspace_bytes, void *stream);

/* ----------------------------------------------------------------------
 * Split-precision tensor-core contractions (the dense T3/T4 residual terms)
 * ---------------------------------------------------------------------- */

/* Index maps below are three-digit mixed radix, f = {R1, R2, S0, S1, S2}:
 *   f(m) = (m / (R1*R2))*S0 + ((m / R2) % R1)*S1 + (m % R2)*S2   (R1, R2 >= 1).
 * A plain stride s is {1, 2^30, 0, 0, s}. */

/* Split an FP64 operand into two K-major pieces, x = hi + lo:
 *   dst[m][k] (m < M, k < Kp; k >= K zero-filled) from src[fm(m) + fk(k)],
 * map10 = {fm, fk} (HOST array).  kind 0: bf16 pieces (Kp multiple of 64),
 * kind 1: tf32 pieces stored as float (Kp multiple of 32).  Replaces the FP64
 * operand of the _einsum calls of distr_cc/rccsdt.py:385-427 (PySCF _einsum
 * backend). */
DCC_API int dcc_split_operand(const double *src, void *hi, void *lo, int64_t M, int64_t K, int64_t Kp,
                              const int64_t *map10, int kind, void *stream);

/* One piece of a K-concatenated operand: columns [k0, k0 + kw) of pieces
 * whose rows are ld elements apart, dst[m][k0 + k] = src[map(m) + map(k)] for
 * k < K and zero for K <= k < kw.  dcc_split_operand is the case k0 = 0,
 * kw = ld = Kp.  Several einsum strings with the same output permutation
 * (distr_cc/rccsdt.py:435-732) become one GEMM over the concatenated K. */
DCC_API int dcc_split_operand_at(const double *src, void *hi, void *lo, int64_t M, int64_t K, int64_t kw,
                                 int64_t ld, int64_t k0, const int64_t *map10, int kind, void *stream);

/* C[frow(m) + fcol(n)] = alpha * (A_hi B_hi + A_hi B_lo + A_lo B_hi)[m][n]
 * + beta * C, FP32 accumulation in tensor memory (tcgen05), FP64 C.  A is
 * [M][Kp], B is [N][Kp] (pieces from dcc_split_operand), epi10 = {frow, fcol}
 * (HOST).  *status (DEVICE int, zero before the call) becomes
 * DCC_ERR_TIMEOUT if a bounded wait gave up.  Replaces the out=..., alpha,
 * beta semantics of the _einsum calls at distr_cc/rccsdt.py:385-427. */
DCC_API int dcc_gemm_split3(const void *A_hi, const void *A_lo, const void *B_hi, const void *B_lo, int64_t M,
                            int64_t N, int64_t Kp, double *C, const int64_t *epi10, double alpha, double beta,
                            int kind, int *status, void *stream);

/* Four-digit address maps, f = {R1, R2, R3, S0, S1, S2, S3}:
 *   f(m) = (m / (R1 R2 R3)) S0 + ((m / (R2 R3)) % R1) S1 + ((m / R3) % R2) S2 + (m % R3) S3,
 * for operands and outputs whose row or column index set folds into four
 * strided digits (the 8-index T4/(Q) blocks of distr_cc/rccsdt_q.py:1014-1129).
 * Same semantics as dcc_split_operand_at / dcc_gemm_split3_ld otherwise;
 * map14 / epi14 hold two such maps (HOST). */
DCC_API int dcc_split_operand_at4(const double *src, void *hi, void *lo, int64_t M, int64_t K, int64_t kw,
                                  int64_t ld, int64_t k0, const int64_t *map14, int kind, void *stream);
/* The same from an FP32 source (the pieces of each value as a double). */
DCC_API int dcc_split_operand_at4_f32(const float *src, void *hi, void *lo, int64_t M, int64_t K, int64_t kw,
                                      int64_t ld, int64_t k0, const int64_t *map14, int kind, void *stream);
DCC_API int dcc_gemm_split3_ld4(const void *A_hi, const void *A_lo, int64_t lda, const void *B_hi, const void *B_lo,
                                int64_t ldb, int64_t M, int64_t N, int64_t Kp, double *C, const int64_t *epi14,
                                double alpha, double beta, int kind, int *status, void *stream);
/* The same into an FP32 C: C[...] = fp32(alpha * acc + beta * C[...]) with the sum taken in FP64
 * (one rounding per store); with beta = 1, C[...] += fp32(alpha * acc) by reductions in L2
 * (red.global.add.f32: no load round trip; each element is written by one thread, so the
 * result is deterministic).  The split precisions keep the residual's intermediate S
 * (the _einsum accumulations of compute_r3_tri, distr_cc/rccsdt.py:385-396, 435-732) in FP32,
 * like the products' own FP32 accumulation, which halves its epilogue traffic. */
DCC_API int dcc_gemm_split3_ld4_f32c(const void *A_hi, const void *A_lo, int64_t lda, const void *B_hi,
                                     const void *B_lo, int64_t ldb, int64_t M, int64_t N, int64_t Kp, float *C,
                                     const int64_t *epi14, double alpha, double beta, int kind, int *status,
                                     void *stream);

/* Grouped split and grouped GEMM: every einsum of one (Q) task group
 * (distr_cc/rccsdt_q.py:390-408, :1014-1129; 132 `_einsum` calls per group,
 * each binding distr_cc/rccsdt_q.py:259) in a handful of launches instead of
 * one split pair and one GEMM per call.
 *
 * dcc_split_grouped_table uploads the parameters of nprob (<= DCC_GROUP_MAX)
 * operand splits to the DEVICE buffer `table` (dcc_split_grouped_table_bytes)
 * and returns their total tile count; spec holds DCC_SPLIT_SPEC int64 values
 * per operand (HOST): hi, lo (device pointers), M, K, kw, ld, k0, map14 (row
 * map then contraction map, four digits each), source type (0 float64,
 * 1 float32).  dcc_split_grouped then fills every operand from its source
 * srcs[p] (HOST array of DEVICE pointers), so one table serves every group
 * of the same shape.
 *
 * dcc_gemm_grouped_table encodes nprob problems C[row(m) + col(n)] +=
 * alpha[p] * (A B^T)[m][n] into the DEVICE buffer `table` (64-byte aligned,
 * dcc_gemm_grouped_table_bytes); spec holds DCC_GEMM_SPEC int64 values per
 * problem (HOST): A_hi, A_lo, lda, B_hi, B_lo, ldb, M, N, Kp, C, output type
 * (0 float64, 1 float32, the same for every problem), epi14, with output
 * offsets below 2^31.  Kp is a multiple of 32 (bf16x3) or 16 (tf32x3);
 * lda / ldb are multiples of 8 and may be below Kp, in which case a row holds
 * only its first lda (ldb) columns and the rest reads as zero.
 * dcc_gemm_grouped runs them all in one persistent launch (out_f32: the
 * table's output type; a mismatch stops the kernel with DCC_ERR_SHAPE in
 * *status); the
 * results are added with reductions in L2, so problems may share C (the
 * summation order between problems is not fixed).  status as for
 * dcc_gemm_split3. */
#define DCC_GROUP_MAX 256
#define DCC_SPLIT_SPEC 22
#define DCC_GEMM_SPEC 25
DCC_API size_t dcc_split_grouped_table_bytes(int nprob);
DCC_API int dcc_split_grouped_table(const int64_t *spec, int nprob, void *table, size_t table_bytes,
                                    int64_t *total_tiles);
DCC_API int dcc_split_grouped(const void *table, int nprob, int64_t total_tiles, const void *const *srcs, int kind,
                              void *stream);
DCC_API size_t dcc_gemm_grouped_table_bytes(int nprob);
DCC_API int dcc_gemm_grouped_table(const int64_t *spec, const double *alpha, int nprob, int kind, void *table,
                                   size_t table_bytes, int64_t *total_tiles);
DCC_API int dcc_gemm_grouped(const void *table, int nprob, int64_t total_tiles, int kind, int out_f32, int *status,
                             void *stream);

/* dcc_gemm_split3 over the first Kp columns of pieces whose rows are lda / ldb
 * elements apart (multiples of 8, >= Kp): one operand of a K-concatenated
 * pair serves a GEMM that needs only its leading piece. */
DCC_API int dcc_gemm_split3_ld(const void *A_hi, const void *A_lo, int64_t lda, const void *B_hi, const void *B_lo,
                               int64_t ldb, int64_t M, int64_t N, int64_t Kp, double *C, const int64_t *epi10,
                               double alpha, double beta, int kind, int *status, void *stream);

/* Pipeline shape of dcc_gemm_split3 (process-wide): bytes of K per k-block
 * (128, 64 or 32 -> matching TMA/UMMA swizzle), ring depth (2 | 3,4 | 8) and
 * the raster group height in M-tiles.  Set by the tile autotuner
 * (dcc.autotune) for each problem shape; no reference counterpart. */
DCC_API int dcc_gemm_set_config(int kb_bytes, int stages, int group_m);
DCC_API int dcc_gemm_get_config(int *kb_bytes, int *stages, int *group_m);
/* The same with the output tile width: tile_n = 256 (128 x 256 tiles, one persistent CTA per
 * SM; the pipelines above) or 128 (128 x 128 tiles, up to two CTAs per SM, 64-byte k-blocks,
 * 2 stages, four epilogue warps, for every K and C type).  dcc_gemm_set_config sets
 * tile_n = 256.  No reference counterpart. */
DCC_API int dcc_gemm_set_tile_config(int kb_bytes, int stages, int group_m, int tile_n);
DCC_API int dcc_gemm_get_tile_config(int *kb_bytes, int *stages, int *group_m, int *tile_n);

#ifdef __cplusplus
}
#endif

#endif /* DCC_B200_H */
