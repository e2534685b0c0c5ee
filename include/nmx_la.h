/*
 * nmx_la.h -- C ABI of the B200-native dense-factorization library
 * (libnmxla.so, sm_100a).
 *
 * This is the boundary numax's Mojo host code binds through `external_call`
 * (or any FFI: ctypes, cffi, a C/C++ caller).  Every entry point takes plain
 * pointers and sizes; matrices are ROW-MAJOR with an explicit leading
 * dimension, exactly as numax's `Tensor.tile()` views are
 * (numax/core/tensor.mojo:636-660).  Pointers named as device pointers must
 * be CUDA device (or managed) memory on the context's device.
 *
 * Return convention (LAPACK-like, numax's `info` semantics):
 *     0        success
 *    <0        -(1-based index of the first invalid argument); nothing was
 *              launched
 *    >0        a factorization's `info` where the entry point documents one
 *              (otherwise info goes to a device word the caller reads)
 *   NMX_ERR_*  a CUDA/runtime failure (large negative codes below)
 * nmx_last_error_string() describes the most recent failure on the calling
 * thread.
 *
 * Asynchrony: every call that takes a `stream` (a cudaStream_t passed as
 * void*) enqueues work on it and returns without synchronizing, unless its
 * comment says otherwise.  numax's calls are synchronous; the wrappers in
 * the Python and Mojo front ends synchronize to keep that behaviour.
 */
#ifndef NMX_LA_H
#define NMX_LA_H

#include <stdint.h>

#if defined(__GNUC__)
#define NMX_API __attribute__((visibility("default")))
#else
#define NMX_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define NMX_ERR_CUDA (-1000)       /* a CUDA runtime call failed */
#define NMX_ERR_ALLOC (-1001)      /* device or host allocation failed */
#define NMX_ERR_UNSUPPORTED (-1002)/* device is not sm_100 / feature absent */
#define NMX_ERR_INTERNAL (-1003)   /* internal error (bounded wait expired, ...) */
#define NMX_ERR_IO (-1004)         /* a file could not be opened, read or written */
#define NMX_ERR_FORMAT (-1005)     /* a file is not what the call asked for */

/* Element types.  The factorizations take NMX_F32 / NMX_F64; the .npy
 * interchange takes every code (NMX_BF16 has no numpy dtype). */
#define NMX_F32 0
#define NMX_F64 1
#define NMX_F16 2
#define NMX_I8 3
#define NMX_I16 4
#define NMX_I32 5
#define NMX_I64 6
#define NMX_U8 7
#define NMX_U16 8
#define NMX_U32 9
#define NMX_U64 10
#define NMX_BOOL 11
#define NMX_BF16 12

typedef struct nmx_context *nmx_ctx;
typedef struct nmx_batched_plan_s *nmx_batched_plan;
typedef struct nmx_syevj_plan_s *nmx_syevj_plan;

/* ---- context ------------------------------------------------------------ */

/* Create a context on CUDA device `device`.  The context owns its workspace
 * and cached plans; it is the stand-in for numax's DeviceContext
 * (numax/core/tensorlike.mojo:116-126).  Not shared across threads without
 * external locking. */
NMX_API int nmx_create(int device, nmx_ctx *out);
NMX_API int nmx_destroy(nmx_ctx ctx);
/* Human-readable description of the last failure on this thread ("" if none). */
NMX_API const char *nmx_last_error_string(void);
/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
NMX_API int nmx_version(void);
/* Wait for everything enqueued on `stream` (numax's ctx.synchronize(), which
 * ends every Tensor-tier call: numax/linalg/lu.mojo:677). */
NMX_API int nmx_synchronize(nmx_ctx ctx, void *stream);
/* Copy `bytes` from device memory to host memory after the work queued on
 * `stream`, and wait for it (how a front end reads an `info` word back to
 * raise numax's message, numax/linalg/cholesky.mojo:385-394). */
NMX_API int nmx_memcpy_to_host(nmx_ctx ctx, void *dst, const void *src, int64_t bytes,
                               void *stream);
/* Per-context tuning knobs, the hook the autotuner writes (0 = automatic):
 *   "lu.leaf_ctas"  CTAs of the cooperative LU leaf panel
 *   "lu.cluster"    cap on the CTAs of the cluster LU leaf (-1 = no cap,
 *                   0 = never use the cluster leaf)
 *   "lu.leaf_w"     widest LU leaf panel in columns (0 = 32; 8..64)
 *   "ir.trsv_ctas"  CTAs of the persistent triangular solves of the IR loop
 *   "ir.tc_min"     smallest inner GEMM dimension the mixed-precision LU
 *                   sends to the tensor cores (-1 = 256; thinner updates
 *                   run in FP32)
 *   "lu.tournament" FP32 panels by tournament pivoting (a stable LU with
 *                   other pivots than numax's): -1 = in the mixed-precision
 *                   LU only, 0 = never, 1 = also in nmx_getrf_f32
 *   "lu.lookahead"  look-ahead panel width of the LU (-1 = 256, from order
 *                   512 with tournament pivoting, from 4096 with numax's
 *                   pivots; 0 = unblocked recursion; 64..1024, <= 512 with
 *                   numax's pivots)
 *   "lu.panel_sms"  SMs the look-ahead keeps free of the update stream's
 *                   tensor-core GEMMs for the panel stream (-1 or 0 = none) */
NMX_API int nmx_tune_set(nmx_ctx ctx, const char *key, int64_t value);
NMX_API int nmx_tune_get(nmx_ctx ctx, const char *key, int64_t *value);

/* ---- batched uneven-size Cholesky + cho_solve ---------------------------
 *
 * Replaces numax's `map_blocks[step=cholesky+cholesky_solve, gpu=True]`
 * (numax/core/functional.mojo:691-834 over the Array-tier bodies
 * numax/linalg/_array/cholesky.mojo:26-92), which runs one fixed-n problem
 * per GPU thread with n <= 64 known at compile time.  Here n varies per
 * matrix (1 <= n_i <= 128) and the batch is one plan.
 *
 * Ragged layout: matrix i is n_i x n_i row-major at element offset
 * a_off[i] = sum_{j<i} n_j^2 of A; its right-hand sides are n_i x nrhs
 * row-major at b_off[i] = sum_{j<i} n_j * nrhs of B and X.
 *
 * Semantics per matrix are the Array tier's: only the lower triangle of A_i
 * is read; l_jj = sqrt(guard_nonzero(d, 1e-30)) (a negative pivot gives NaN,
 * an exactly-zero one 1e-15); solves divide by guard_nonzero(l_ii, 1e-30).
 * On return the lower triangle of L_i holds the factor (the upper triangle
 * of L_i is not written; L may alias A for an in-place factorization),
 * X_i = A_i^-1 B_i, and info[i] is the 1-based index of the first pivot
 * d <= 0 (0 if none) -- the `info` rule of numax's potrf_diag
 * (numax/linalg/panel.mojo:216-286), which the Array tier lacks.
 */

/* Build a plan: sorts the batch by size into buckets (n <= 32, 64, 96, 128),
 * gives each bucket its default CTA shape and uploads the schedule: the
 * 8 x 8 DMMA tile kernel with 1 warp per matrix up to n = 64, 2 up to 96 and
 * 4 up to 128 (it computes in FP64; an NMX_F32 batch is widened on load and
 * L, X rounded to FP32 on store).
 * nmx_batched_plan_autotune / _set_shape change the shapes.  n_host: count
 * sizes on the HOST.  dtype: NMX_F32 / NMX_F64.  nrhs: 0..8. */
NMX_API int nmx_potrf_potrs_batched_plan(nmx_ctx ctx, int dtype, int64_t count, const int32_t *n_host,
                                 int nrhs, nmx_batched_plan *out);
NMX_API int nmx_batched_plan_destroy(nmx_batched_plan plan);
/* Elements of A (sum n_i^2) and of B/X (sum n_i*nrhs) the plan expects. */
NMX_API int nmx_batched_plan_sizes(nmx_batched_plan plan, int64_t *a_elems, int64_t *b_elems);

/* Run the plan on device buffers.  A and B are read; L (lower triangles),
 * X and info (count int32) are written.  L may alias A, X may alias B. */
NMX_API int nmx_potrf_potrs_batched_f64(nmx_ctx ctx, nmx_batched_plan plan, const double *A,
                                        double *L, const double *B, double *X, int32_t *info,
                                        void *stream);
NMX_API int nmx_potrf_potrs_batched_f32(nmx_ctx ctx, nmx_batched_plan plan, const float *A,
                                        float *L, const float *B, float *X, int32_t *info,
                                        void *stream);

/* Autotuner (no numax counterpart; numax launches one problem per thread at
 * a compile-time n): times every CTA shape (64, 96, 128, 192 threads of the
 * packed-triangle kernel, and the kernel on 8 x 8 DMMA tiles with 1, 2, 4
 * or 8 warps per matrix, shapes NMX_BATCHED_TILE_SHAPE(warps)) that
 * covers each size bucket of the plan on these buffers -- the bucket's
 * persistent kernel alone, best of `reps` runs, CUDA events -- and keeps the
 * fastest in the plan.  Every run computes the whole bucket, so L, X and
 * info hold a valid result afterwards.  A and B as for the run entry points
 * of the plan's dtype.  Synchronizes `stream`.  reps: 1..100. */
NMX_API int nmx_batched_plan_autotune(nmx_ctx ctx, nmx_batched_plan plan, const void *A, void *L,
                                      const void *B, void *X, int32_t *info, int reps,
                                      void *stream);
/* The plan's schedule: per bucket (largest n first) its largest n, CTA
 * shape (threads per CTA of the packed-triangle kernel, or
 * NMX_BATCHED_TILE_SHAPE(warps)) and CTAs launched; up to max_buckets
 * entries, *nbuckets = count. */
#define NMX_BATCHED_TILE_SHAPE(warps) (1000 + 32 * (warps))
NMX_API int nmx_batched_plan_schedule(nmx_batched_plan plan, int32_t *nmax, int32_t *threads,
                                      int32_t *ctas, int max_buckets, int32_t *nbuckets);
/* Split one ragged batch over `ndev` devices by predicted cost (host only, no
 * device needed): dev_of[i] receives the device of matrix i, cost_per_dev
 * (may be NULL) each device's total.  The cost of a matrix is its flops
 * (n^3/3 + 2 nrhs n^2) plus its n^2-element read and write weighted at the
 * B200's FP64 / HBM balance; matrices go largest first to the least-loaded
 * device (longest processing time first, deterministic ties).  Each device
 * then builds its own plan over its share: no data moves between devices.
 * No numax counterpart (numax runs on one device). */
NMX_API int nmx_batched_partition(int64_t count, const int32_t *n_host, int nrhs, int ndev,
                                  int32_t *dev_of, double *cost_per_dev);
/* Set the CTA shape of one size bucket (bucket >= 0) or of all (-1) by hand,
 * in place of the default or the autotuner's pick (no numax counterpart):
 * threads 64, 96, 128 or 192 select the packed-triangle kernel,
 * NMX_BATCHED_TILE_SHAPE(1, 2, 4 or 8) = 1032, 1064, 1128 or 1256 the
 * kernel on 8 x 8 DMMA tiles with that many warps per matrix.  Rejects a
 * shape that cannot cover a bucket or does not fit an SM. */
NMX_API int nmx_batched_plan_set_shape(nmx_ctx ctx, nmx_batched_plan plan, int bucket,
                                       int threads);
/* Run the plan through a CUDA graph (no numax counterpart): the first call
 * with a given set of buffers captures the plan's launches (counter reset +
 * one persistent kernel per bucket) on an internal stream into a graph kept
 * in the plan; later calls with the same buffers replay it on `stream` with
 * one launch.  New buffers or an autotune re-capture. */
NMX_API int nmx_potrf_potrs_batched_graph_f64(nmx_ctx ctx, nmx_batched_plan plan, const double *A,
                                              double *L, const double *B, double *X,
                                              int32_t *info, void *stream);
NMX_API int nmx_potrf_potrs_batched_graph_f32(nmx_ctx ctx, nmx_batched_plan plan, const float *A,
                                              float *L, const float *B, float *X, int32_t *info,
                                              void *stream);

/* Allocation-free form of nmx_potrf_potrs_batched_f64, with no counterpart
 * in the reference (numax allocates per call).  For callers that cannot
 * allocate device memory -- a host runtime whose allocator already owns the
 * GPU's memory, or code running inside another framework's memory pool --
 * the batch's schedule (sizes, size-sorted order, offsets, work counter) is
 * kept in a fixed device array built into the library instead of a plan's
 * cudaMalloc'd buffer.  The call itself allocates nothing on the device or
 * through any library.  Same layout and results as the plan path; n_host is
 * on the host, its sizes are checked there, and it is copied into that array
 * on `stream`.  From pageable memory the copy is staged before the call
 * returns, so n_host may be reused at once; from pinned memory the copy is
 * asynchronous, so keep n_host unchanged until `stream` has passed the call.
 * Limit: count <= 65536 matrices (a larger count is rejected with -2).
 * The array (about 1.5 MB) stays resident on every GPU that loads the
 * library until exit.  The first call on a device performs that device's
 * set-up (resolving the array's address), so make it before any stream
 * capture.  A call whose `stream` is being captured is refused with
 * NMX_ERR_UNSUPPORTED, because the size checks happen on the host at call
 * time.  All calls share the one array: calls that may overlap on the GPU
 * (different streams, or several host threads) race and must be serialized
 * by the caller. */
NMX_API int nmx_potrf_potrs_batched_noalloc_f64(nmx_ctx ctx, int64_t count, const int32_t *n_host,
                                                int nrhs, const double *A, double *L,
                                                const double *B, double *X, int32_t *info,
                                                void *stream);

/* ---- batched uneven-size symmetric eigensolver (Jacobi) -----------------
 *
 * Replaces numax's Array-tier `eigh[T, n, sweeps=12]` run one matrix per GPU
 * thread (numax/linalg/_array/eigen.mojo:316-392; launched through `map` in
 * examples/advanced/quantum_well.mojo:149-157).  float32 data, float64
 * rotation angles (numax's formula, numax/linalg/_array/eigen.mojo:34-75)
 * and a float64 off-diagonal-norm stopping test.  Parallel (round-robin)
 * ordering replaces numax's cyclic order, so eigenvalues agree to rounding
 * but their unsorted order may differ; `sort` = 1 returns them ascending
 * with V's columns permuted to match (numpy.linalg.eigh's order).
 *
 * Ragged layout: A_i and V_i are n_i x n_i row-major at a_off[i] = sum n_j^2;
 * W_i (n_i values) at w_off[i] = sum n_j.  1 <= n_i <= 64.  The whole matrix
 * is read (numax's eigh assumes symmetry and does not check it).  V's columns
 * are the eigenvectors.  sweeps[i] (optional, may be NULL) receives the
 * number of sweeps run.  A sweep runs while off(A) > tol * ||A||_F and fewer
 * than max_sweeps sweeps have run.
 */
NMX_API int nmx_syevj_batched_plan(nmx_ctx ctx, int64_t count, const int32_t *n_host,
                                   nmx_syevj_plan *out);
NMX_API int nmx_syevj_plan_destroy(nmx_syevj_plan plan);
NMX_API int nmx_syevj_plan_sizes(nmx_syevj_plan plan, int64_t *a_elems, int64_t *w_elems);
NMX_API int nmx_syevj_batched_f32(nmx_ctx ctx, nmx_syevj_plan plan, const float *A, float *W,
                                  float *V, int32_t *sweeps, double tol, int max_sweeps, int sort,
                                  void *stream);
/* Autotuner (no numax counterpart): times every (threads, group) shape --
 * a warp per matrix in CTAs of 1, 2, 4 or 8 warps, or a CTA of 64, 128 or
 * 256 threads per matrix -- on each size bucket with these buffers and
 * arguments (best of `reps`, CUDA events) and keeps the fastest; then runs
 * the kept schedule once, so W, V and sweeps hold its result.  Synchronizes. */
NMX_API int nmx_syevj_plan_autotune(nmx_ctx ctx, nmx_syevj_plan plan, const float *A, float *W,
                                    float *V, int32_t *sweeps, double tol, int max_sweeps,
                                    int sort, int reps, void *stream);
/* Per bucket (largest n first): its largest n, threads per CTA, threads per
 * matrix (group) and CTAs launched. */
NMX_API int nmx_syevj_plan_schedule(nmx_syevj_plan plan, int32_t *nmax, int32_t *threads,
                                    int32_t *group, int32_t *ctas, int max_buckets,
                                    int32_t *nbuckets);
/* nmx_syevj_batched_f32 through a CUDA graph of the plan's launches (counter
 * reset and one persistent kernel per bucket), captured on an internal
 * stream the first time these buffers and arguments are seen and replayed on
 * `stream` after that; an autotune or new arguments re-capture. */
NMX_API int nmx_syevj_batched_graph_f32(nmx_ctx ctx, nmx_syevj_plan plan, const float *A, float *W,
                                        float *V, int32_t *sweeps, double tol, int max_sweeps,
                                        int sort, void *stream);

/* ---- dense LU with partial pivoting, and its solve ----------------------
 *
 * nmx_getrf_*: factor the n x n row-major A (leading dimension lda) in place
 * into P L U -- numax's lu_factor (numax/linalg/lu.mojo:454-701) with its
 * getrf2 recursive panel (numax/linalg/panel.mojo:445-586) taken over the
 * whole matrix.  On return A holds L strictly below the diagonal (unit
 * diagonal implicit) and U on and above it; ipiv[j] (0-based, device int32)
 * is the row interchanged with row j, applied across the full width in
 * order (numax/linalg/lu.mojo:114-122); *info (device int32) is the 1-based
 * index of the first column with no nonzero pivot candidate, 0 otherwise.
 * The pivot rule is numax's: largest |a|, the lowest row on ties
 * (numax/linalg/panel.mojo:350-388).  A zero pivot is floored to 1e-30 for
 * the division and the factorization continues, so a singular A yields
 * non-finite solves rather than an error (numax/linalg/lu.mojo:96-98).
 *
 * nmx_getrs_*: B := A^-1 B for the n x nrhs row-major B (ldb), from the
 * factors: interchanges, unit-lower solve, upper solve -- numax's LU.solve
 * (numax/linalg/lu.mojo:181-354).
 */
NMX_API int nmx_getrf_f64(nmx_ctx ctx, int64_t n, double *A, int64_t lda, int32_t *ipiv,
                          int32_t *info, void *stream);
NMX_API int nmx_getrf_f32(nmx_ctx ctx, int64_t n, float *A, int64_t lda, int32_t *ipiv,
                          int32_t *info, void *stream);
NMX_API int nmx_getrs_f64(nmx_ctx ctx, int64_t n, int64_t nrhs, const double *LU, int64_t lda,
                          const int32_t *ipiv, double *B, int64_t ldb, void *stream);
NMX_API int nmx_getrs_f32(nmx_ctx ctx, int64_t n, int64_t nrhs, const float *LU, int64_t lda,
                          const int32_t *ipiv, float *B, int64_t ldb, void *stream);

/* ---- dense Cholesky and its solve ----------------------------------------
 *
 * nmx_potrf_*: factor the SPD n x n row-major A (lda) in place into L L^T,
 * reading only the lower triangle -- numax's cholesky
 * (numax/linalg/cholesky.mojo:59-396) with potrf_diag's failure rule
 * (numax/linalg/panel.mojo:216-286): a pivot d <= 0 is floored to 1e-30 and
 * the factorization continues; *info (device int32) receives the 1-based
 * index of the first such pivot, 0 if none.  On return the lower triangle
 * holds L and the upper triangle is zeroed (numax's `tril`,
 * numax/linalg/cholesky.mojo:396).  numax raises "cholesky: matrix is not
 * positive definite (non-positive pivot at index i)" with i = info - 1; the
 * front ends reproduce that from info.
 *
 * nmx_potrs_*: B := A^-1 B from L: L y = b, then L^T x = y reading L in place
 * (numax's cholesky_solve, numax/linalg/cholesky.mojo:471-580).
 */
NMX_API int nmx_potrf_f64(nmx_ctx ctx, int64_t n, double *A, int64_t lda, int32_t *info,
                          void *stream);
NMX_API int nmx_potrf_f32(nmx_ctx ctx, int64_t n, float *A, int64_t lda, int32_t *info,
                          void *stream);
NMX_API int nmx_potrs_f64(nmx_ctx ctx, int64_t n, int64_t nrhs, const double *L, int64_t lda,
                          double *B, int64_t ldb, void *stream);
NMX_API int nmx_potrs_f32(nmx_ctx ctx, int64_t n, int64_t nrhs, const float *L, int64_t lda,
                          float *B, int64_t ldb, void *stream);

/* ---- what an LU gives besides solves -------------------------------------
 *
 * nmx_lu_slogdet_*: from nmx_getrf's packed factor and pivots, out[0] = sign,
 * out[1] = ln|det|, out[2] = det (device pointer, 3 values; asynchronous):
 * numax's LU.slogdet / LU.det (numax/linalg/lu.mojo:382-451) -- sign = swap
 * parity x the signs of U's diagonal, (0, -inf) and det 0 when a diagonal
 * entry is exactly 0, det = parity x the diagonal multiplied in index order.
 * nmx_lu_unpack_*: numax's lu -> PLU (numax/linalg/lu.mojo:877-975): A = P L U
 * with L unit lower, U upper and P[perm[i]][i] = 1, perm the interchanges
 * replayed on the identity; any of P, L, U may be NULL.
 * nmx_inverse_*: numax's inverse (numax/linalg/basic.mojo:149-192): X =
 * A^-1 by one LU of a copy of A (ipiv: n device int32, info as nmx_getrf)
 * and one solve against the identity; a singular A gives non-finite entries,
 * as numax's does, with info > 0.
 */
NMX_API int nmx_lu_slogdet_f64(nmx_ctx ctx, int64_t n, const double *LU, int64_t lda,
                               const int32_t *ipiv, double *out, void *stream);
NMX_API int nmx_lu_slogdet_f32(nmx_ctx ctx, int64_t n, const float *LU, int64_t lda,
                               const int32_t *ipiv, float *out, void *stream);
NMX_API int nmx_lu_unpack_f64(nmx_ctx ctx, int64_t n, const double *LU, int64_t lda,
                              const int32_t *ipiv, double *P, int64_t ldp, double *L, int64_t ldl,
                              double *U, int64_t ldu, void *stream);
NMX_API int nmx_lu_unpack_f32(nmx_ctx ctx, int64_t n, const float *LU, int64_t lda,
                              const int32_t *ipiv, float *P, int64_t ldp, float *L, int64_t ldl,
                              float *U, int64_t ldu, void *stream);
NMX_API int nmx_inverse_f64(nmx_ctx ctx, int64_t n, const double *A, int64_t lda, double *X,
                            int64_t ldx, int32_t *ipiv, int32_t *info, void *stream);
NMX_API int nmx_inverse_f32(nmx_ctx ctx, int64_t n, const float *A, int64_t lda, float *X,
                            int64_t ldx, int32_t *ipiv, int32_t *info, void *stream);

/* ---- Householder QR (m >= n) and the thin Q --------------------------------
 *
 * nmx_geqrf_*: factor the m x n row-major A (lda) in place into LAPACK's
 * packed form -- R on and above the diagonal of the first n rows, each
 * reflector's v below the diagonal with an implicit unit leading entry, its
 * scale in tau[j] -- numax's qr_factor (numax/linalg/qr.mojo:615-743) with
 * geqr2_panel's convention (numax/linalg/panel.mojo:1975-2073):
 * beta = -sign(alpha)*||x|| (+||x|| when alpha <= 0), tau = (beta-alpha)/beta,
 * v = x/(alpha-beta), tau = 0 for an exactly zero sub-column.  Panels are 16
 * columns, numax's default block.
 *
 * nmx_orgqr_*: the thin Q (m x n, row-major ldq) from geqrf's output F and
 * tau, the reflectors replayed last panel first on the identity -- numax's
 * QR.q() (numax/linalg/qr.mojo:405-468).
 */
NMX_API int nmx_geqrf_f32(nmx_ctx ctx, int64_t m, int64_t n, float *A, int64_t lda, float *tau,
                          void *stream);
NMX_API int nmx_geqrf_f64(nmx_ctx ctx, int64_t m, int64_t n, double *A, int64_t lda, double *tau,
                          void *stream);
NMX_API int nmx_orgqr_f32(nmx_ctx ctx, int64_t m, int64_t n, const float *F, int64_t ldf,
                          const float *tau, float *Q, int64_t ldq, void *stream);
NMX_API int nmx_orgqr_f64(nmx_ctx ctx, int64_t m, int64_t n, const double *F, int64_t ldf,
                          const double *tau, double *Q, int64_t ldq, void *stream);
/* nmx_ormqr_*: B := Q^T B in place for the m x nrhs row-major B (ldb), Q the
 * full orthogonal factor of geqrf's output, never formed -- numax's
 * QR.apply_q_transpose (numax/linalg/qr.mojo:470-530): the panels' block
 * reflectors in factorization order.  The leading n rows are the thin Q^T B.
 * nmx_qr_solve_*: x (n) = the least-squares solution of A x ~= b (m) from
 * geqrf's output -- numax's QR.solve / lstsq (numax/linalg/qr.mojo:532-612):
 * Q^T b (in `work`, m values, device) then the back substitution with R.
 * Rank deficiency is not detected, as in numax. */
NMX_API int nmx_ormqr_f32(nmx_ctx ctx, int64_t m, int64_t n, const float *F, int64_t ldf,
                          const float *tau, float *B, int64_t ldb, int64_t nrhs, void *stream);
NMX_API int nmx_ormqr_f64(nmx_ctx ctx, int64_t m, int64_t n, const double *F, int64_t ldf,
                          const double *tau, double *B, int64_t ldb, int64_t nrhs, void *stream);
NMX_API int nmx_qr_solve_f32(nmx_ctx ctx, int64_t m, int64_t n, const float *F, int64_t ldf,
                             const float *tau, const float *b, float *x, float *work,
                             void *stream);
NMX_API int nmx_qr_solve_f64(nmx_ctx ctx, int64_t m, int64_t n, const double *F, int64_t ldf,
                             const double *tau, const double *b, double *x, double *work,
                             void *stream);

/* ---- the dense factorizations' GEMM ---------------------------------------
 *
 * C = alpha op(A) op(B) + beta C, row-major with leading dimensions, op(X) =
 * X or X^T (trans_a / trans_b nonzero); `lower` nonzero writes only C's lower
 * triangle (column <= row) and skips the tiles above it (the SYRK-shaped
 * update).  beta == 0 never reads C.  FP64 runs on the DMMA pipe, FP32 on the
 * CUDA cores, both hand-written.  The updates numax runs through MAX's
 * linalg.matmul: numax/linalg/lu.mojo:646-673 (A22 -= L21 U12),
 * numax/linalg/cholesky.mojo:190-225 (A22 -= L21 L21^T), the triangular
 * solves' block products (numax/linalg/triangular.mojo:193-218) and the
 * block-reflector products (numax/linalg/qr.mojo:262-308).  Asynchronous on
 * `stream`.
 */
NMX_API int nmx_gemm_f64(nmx_ctx ctx, int trans_a, int trans_b, int64_t m, int64_t n, int64_t k,
                         double alpha, const double *A, int64_t lda, const double *B, int64_t ldb,
                         double beta, double *C, int64_t ldc, int lower, void *stream);
NMX_API int nmx_gemm_f32(nmx_ctx ctx, int trans_a, int trans_b, int64_t m, int64_t n, int64_t k,
                         float alpha, const float *A, int64_t lda, const float *B, int64_t ldb,
                         float beta, float *C, int64_t ldc, int lower, void *stream);

/* ---- mixed-precision LU solve with iterative refinement -------------------
 *
 * No numax counterpart (numax's GPU path is FP32-only, without refinement);
 * the north star's large solve.  x := A^-1 b for the FP64 n x n row-major A
 * (lda) and FP64 vectors b, x (device):
 *   - A is scaled by powers of two (rows, then columns; exact) when the
 *     factors are FP16, rounded to FP32 and factored by the recursive LU of
 *     nmx_getrf_f32 with its trailing updates in BF16/FP16 on the tcgen05
 *     tensor cores (FP32 accumulate), or FP32 CUDA cores (NMX_IR_FP32);
 *     NMX_IR_FP64 factors A in FP64 (nmx_getrf_f64) and only polishes;
 *   - refinement in FP64: r = b - A x over the original A, correction from
 *     the low-precision factors; with NMX_IR_GMRES the correction is solved by
 *     GMRES preconditioned by those factors (GMRES-IR, on the device); with
 *     NMX_IR_AUTO plain refinement hands over to GMRES-IR when it stops
 *     contracting; with NMX_IR_ESCALATE a precision whose refinement cannot
 *     converge is replaced by the next, more accurate one (BF16 or FP16 ->
 *     BF16X3 -> BF16X6 -> FP64), refining on from the best iterate.
 * x receives the iterate with the smallest backward error.  Stops when
 * ||b - A x||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= tol or after max_iter
 * refinement steps.  Synchronizes `stream` (the refinement loop decides on the
 * host).  stats (host pointer, may be NULL) receives the iteration counts,
 * the final normwise backward error, the device time of the factorizations
 * and of the refinement, and the precision the last factorization used.
 * Workspace is grown on first use; nmx_gesv_ir_reserve grows it ahead.
 */
#define NMX_IR_BF16 1
#define NMX_IR_FP16 2
#define NMX_IR_FP32 3
#define NMX_IR_BF16X3 4 /* BF16 tensor cores on hi/lo splits (see NMX_PREC_BF16X3) */
#define NMX_IR_BF16X6 5 /* BF16 tensor cores on hi/mid/lo splits (see NMX_PREC_BF16X6) */
#define NMX_IR_FP64 6   /* FP64 factors: the last escalation level */
#define NMX_IR_GMRES 0x10
#define NMX_IR_AUTO 0x20
#define NMX_IR_ESCALATE 0x40

typedef struct {
    int32_t iterations;       /* refinement steps taken */
    int32_t gmres_iterations; /* total inner GMRES iterations */
    int32_t converged;        /* 1 if the backward error reached tol */
    int32_t info;             /* info of the low-precision LU (first zero pivot) */
    int32_t used_gmres;       /* 1 if GMRES-IR ran */
    int32_t final_precision;  /* NMX_IR_* precision of the last factorization */
    double backward_error;    /* final normwise backward error */
    double factor_ms;         /* device time: scaling + low-precision LU */
    double refine_ms;         /* device time: the refinement loop */
} nmx_ir_stats;

/* The trailing-update primitive of the mixed-precision factorizations on its
 * own: C[M x N] -= round(A)[M x K] * round(B)[K x N] for fp32 row-major
 * operands, A and B rounded to BF16 (precision 1) or FP16 (precision 2) and
 * the products accumulated in FP32 on the tcgen05 tensor cores.  Precision 3
 * (BF16X3) splits each operand into BF16 hi + lo (lo = the rounding
 * residual) and forms hi*hi + hi*lo + lo*hi as one BF16 GEMM over 3K: about
 * 16 significant bits per operand instead of 8; precision 4 (BF16X6) splits
 * into hi + mid + lo and forms the six products hi*hi, hi*mid, mid*hi,
 * hi*lo, mid*mid, lo*hi over 6K: FP32's 24 bits.  C must be
 * 16-byte aligned with ldc a multiple of 4 and ldc >= N rounded up to 8: the
 * update runs on N (and K) rounded up to 8 with zero padding, so C's columns
 * N .. round8(N)-1 are read and written back unchanged.  No numax
 * counterpart (the role MAX's matmul plays in numax/linalg/lu.mojo:646-673). */
#define NMX_PREC_BF16 1
#define NMX_PREC_FP16 2
#define NMX_PREC_BF16X3 3
#define NMX_PREC_BF16X6 4
NMX_API int nmx_gemm_sub_f32(nmx_ctx ctx, int64_t M, int64_t N, int64_t K, const float *A,
                             int64_t lda, const float *B, int64_t ldb, float *C, int64_t ldc,
                             int precision, void *stream);

NMX_API int nmx_gesv_ir_f64(nmx_ctx ctx, int64_t n, const double *A, int64_t lda, const double *b,
                            double *x, int mode, double tol, int max_iter, nmx_ir_stats *stats,
                            void *stream);
/* Grow the context's workspace for nmx_gesv_ir_f64 at order n and `mode`
 * (with NMX_IR_ESCALATE, for every level it may reach) so that the solve
 * itself allocates nothing.  No numax counterpart. */
NMX_API int nmx_gesv_ir_reserve(nmx_ctx ctx, int64_t n, int mode);

/* Mixed-precision Cholesky solve with iterative refinement: nmx_gesv_ir_f64's
 * scheme for a symmetric positive definite A.  A is scaled symmetrically by
 * powers of two (D A D, diagonal near 1), rounded to FP32 and factored by the
 * recursive Cholesky of nmx_potrf_f32 with its SYRK and triangular-solve
 * products on the tcgen05 tensor cores in the mode's precision; the
 * corrections come from D L^-T L^-1 D, the residual and every other step as
 * in nmx_gesv_ir_f64 (GMRES-IR, escalation up to an FP64 Cholesky, the best
 * iterate returned).  The factorization reads A's lower triangle, the FP64
 * residual all of A: both triangles must hold the matrix.  No numax
 * counterpart; extends numax's cholesky (numax/linalg/cholesky.mojo:59-230)
 * to low-precision factors with FP64 accuracy. */
NMX_API int nmx_posv_ir_f64(nmx_ctx ctx, int64_t n, const double *A, int64_t lda, const double *b,
                            double *x, int mode, double tol, int max_iter, nmx_ir_stats *stats,
                            void *stream);
NMX_API int nmx_posv_ir_reserve(nmx_ctx ctx, int64_t n, int mode);

/* ---- symmetric eigendecomposition of one matrix --------------------------
 *
 * nmx_syevd_*: the eigenvalues (W, n, ascending) and, when V is not NULL,
 * orthonormal eigenvectors (V's columns, row-major ldv, V[:, j] for W[j]) of
 * the symmetric n x n row-major A (lda), reading only its lower triangle --
 * numax's Tensor-tier eigh (numax/linalg/eigen.mojo:1268-1341); with
 * V = NULL, numax's eigvalsh.  A is not modified.  The work is FP64 in both
 * entry points (the FP32 one rounds its outputs): a Householder
 * tridiagonalization in one cooperative launch, then Sturm bisection
 * (values only) or divide and conquer on the tridiagonal, then the
 * reflectors applied to the tridiagonal's eigenvectors.  *info (device
 * int32) is 1 when A's lower triangle holds a NaN or an infinity (numax
 * raises that its QL sweep did not converge), else 0; W and V are then
 * filled with NaN.  Synchronous: returns after the work on `stream` is done
 * (the divide and conquer sizes its products from counts it reads back).
 * Order limit: n - 1 <= 8 x 16 x (SM count), 18,944 on a B200; the device
 * workspace is about 5 n^2 doubles with vectors, n^2 without.
 */
NMX_API int nmx_syevd_f64(nmx_ctx ctx, int64_t n, const double *A, int64_t lda, double *W,
                          double *V, int64_t ldv, int32_t *info, void *stream);
NMX_API int nmx_syevd_f32(nmx_ctx ctx, int64_t n, const float *A, int64_t lda, float *W, float *V,
                          int64_t ldv, int32_t *info, void *stream);

/* ---- .npy interchange ----------------------------------------------------
 *
 * Replaces numax's `numpy.save` / `numpy.load` / `numpy.load_dyn`
 * (numax/io/npy.mojo:273-453): read what numpy.save wrote, write what
 * numpy.load reads, format versions 1.0 and 2.0.  The payload is C order, so a
 * (count, n, n) stack of matrices saved by numpy is already the batched
 * entry points' layout (A_i at i * n * n) and loads into it with no host-side
 * transpose; a ragged batch is a 1-D file of the matrices back to back.
 *
 * With ctx != NULL the array lives in device memory on ctx's device and the
 * payload streams through pinned staging buffers kept in the context:
 * worker threads read (write) fixed-size chunks of the file while earlier
 * chunks are copied to (from) the device on `stream`.  With ctx == NULL the
 * array is host memory and no CUDA call is made.  Both calls return when the
 * data has landed (numax's calls are synchronous).
 *
 * Rejected, with numax's messages (nmx_last_error_string) and
 * NMX_ERR_FORMAT: a file without the .npy magic (an .npz archive), format
 * versions other than 1.x / 2.x, a truncated header, Fortran order, a
 * big-endian descr, a descr naming another element type, a payload length
 * that disagrees with the header, a rank or an extent other than the
 * requested ones (npy.mojo:138-260, 349-453).  NMX_ERR_IO when the file
 * cannot be opened, read or written.
 */
#define NMX_NPY_MAX_RANK 64
/* The header of `path`: *dtype the NMX_* code its descr names (-1 when it
 * names none of them), *rank, shape[0 .. rank) (room for max_rank entries),
 * *payload_offset where the payload starts.  Any output may be NULL except
 * shape when the file's rank is above 0. */
NMX_API int nmx_npy_header(const char *path, int *dtype, int *rank, int64_t *shape, int max_rank,
                           int64_t *payload_offset);
/* Load `path` into `dst` (dst_bytes of room).  The file must hold `dtype`
 * at rank `rank`; shape[i] >= 0 must equal the file's extent i (numax's
 * `load`), shape[i] = -1 accepts any extent (numax's `load_dyn`).  On
 * success shape[] holds the file's extents. */
NMX_API int nmx_npy_load(nmx_ctx ctx, const char *path, int dtype, int rank, int64_t *shape,
                         void *dst, int64_t dst_bytes, void *stream);
/* Write the C-order array `src` (dtype, rank, shape) to `path`, the bytes
 * numpy.save writes for it: the sorted-key header dict, numpy's spare space
 * after it, padding to 64 bytes, the payload.  With ctx != NULL the copy
 * out follows the work already queued on `stream`. */
NMX_API int nmx_npy_save(nmx_ctx ctx, const char *path, int dtype, int rank,
                         const int64_t *shape, const void *src, void *stream);

#ifdef __cplusplus
}
#endif

#endif /* NMX_LA_H */
