// Building blocks shared by the dense factorizations (LU, Cholesky, QR):
// the cooperative grid barrier with a bounded wait, the trailing-update GEMM
// dispatch, row interchanges and small triangular solves.  Row-major storage
// with a leading dimension throughout, as numax's Tensor tiles are.
#pragma once

#include "gemm_cc.cuh"
#include "gemm_tc.cuh"
#include "nmx_common.cuh"

namespace nmx {

// Grid-wide barrier for cooperative launches.  `bar` counts arrivals and is
// zeroed before the launch; barrier number `gen` (0, 1, ...) completes when
// all `nctas` have arrived gen+1 times.  The wait is bounded: after
// kSpinLimit polls it sets *err and reports failure so the kernel can
// return instead of hanging.
constexpr long long kSpinLimit = 1ll << 26;

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// Returns false (for every thread of the CTA) if the wait gave up.
__device__ __forceinline__ bool grid_barrier(unsigned *bar, unsigned gen, unsigned nctas, int *err,
                                             int *s_flag) {
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
        const unsigned target = (gen + 1) * nctas;
        long long spins = 0;
        int ok = 1;
        while (ld_acquire(bar) < target) {
            if (++spins > kSpinLimit) {
                atomicExch(err, 1);
                ok = 0;
                break;
            }
            if (spins > 64) __nanosleep(64);
        }
        __threadfence();
        *s_flag = ok;
    }
    __syncthreads();
    return *s_flag != 0;
}

// C[m x n] -= A[m x k] * B[k x n], all row-major with leading dimensions,
// on the library's own FP64 (DMMA) / FP32 (FFMA) GEMM.
template <typename T>
inline int gemm_sub(cudaStream_t st, int64_t m, int64_t n, int64_t k, const T *A, int64_t lda,
                    const T *B, int64_t ldb, T *C, int64_t ldc) {
    if (m <= 0 || n <= 0 || k <= 0) return 0;
    return gemm_cc<T>(st, false, false, m, n, k, T(-1), A, lda, B, ldb, T(1), C, ldc);
}

// C[m x n] -= A[m x k] * B[n x k]^T (row-major).  `lower`: only C's lower
// triangle (the SYRK-shaped update with B = A).
template <typename T>
inline int gemm_sub_bt(cudaStream_t st, int64_t m, int64_t n, int64_t k, const T *A, int64_t lda,
                       const T *B, int64_t ldb, T *C, int64_t ldc, bool lower = false) {
    if (m <= 0 || n <= 0 || k <= 0) return 0;
    return gemm_cc<T>(st, false, true, m, n, k, T(-1), A, lda, B, ldb, T(1), C, ldc, lower);
}

// Creates the context's look-ahead streams and events on first use.
int ctx_lookahead_streams(nmx_ctx ctx);


// The trailing-update product of the recursive factorizations and solves:
// C[m x n] -= A[m x k] B[k x n], row-major.  precision 0 keeps the operands'
// own precision (the DMMA / FFMA GEMM of gemm_cc.cu); NMX_PREC_BF16 /
// NMX_PREC_FP16 / NMX_PREC_BF16X3 (fp32 data only) round or split the
// operands to 16 bits and run the tcgen05 kernel.
struct GemmSub {
    cudaStream_t st = nullptr;
    int precision = 0;
    int64_t tc_min = 256;
    void *ws = nullptr;
    size_t ws_bytes = 0;
    int sm_limit = 0;  // > 0: tensor-core updates on at most this many SMs
    int operator()(int64_t m, int64_t n, int64_t k, const double *A, int64_t lda, const double *B,
                   int64_t ldb, double *C, int64_t ldc) const {
        return gemm_sub<double>(st, m, n, k, A, lda, B, ldb, C, ldc);
    }
    int operator()(int64_t m, int64_t n, int64_t k, const float *A, int64_t lda, const float *B,
                   int64_t ldb, float *C, int64_t ldc) const {
        // Tensor cores for the updates with both inner dimensions >= tc_min;
        // the thin ones near the recursion's leaves stay FP32 (their operand
        // rounding passes and launches would cost more than they save).
        if (precision && n >= tc_min && k >= tc_min)
            return tc_gemm_sub_f32(st, precision, m, n, k, A, lda, B, ldb, C, ldc, ws, ws_bytes,
                                   sm_limit);
        return gemm_sub<float>(st, m, n, k, A, lda, B, ldb, C, ldc);
    }
    // C[m x n] -= A[m x k] B[n x k]^T; `lower`: only C's lower triangle is
    // needed (the SYRK-shaped update; the tensor-core path writes all of C,
    // so its strict upper triangle must be scratch).
    int sub_bt(int64_t m, int64_t n, int64_t k, const double *A, int64_t lda, const double *B,
               int64_t ldb, double *C, int64_t ldc, bool lower = false) const {
        return gemm_sub_bt<double>(st, m, n, k, A, lda, B, ldb, C, ldc, lower);
    }
    int sub_bt(int64_t m, int64_t n, int64_t k, const float *A, int64_t lda, const float *B,
               int64_t ldb, float *C, int64_t ldc, bool lower = false) const {
        if (precision && n >= tc_min && k >= tc_min)
            return tc_gemm_sub_bt_f32(st, precision, m, n, k, A, lda, B, ldb, C, ldc, ws, ws_bytes);
        return gemm_sub_bt<float>(st, m, n, k, A, lda, B, ldb, C, ldc, lower);
    }
};

// Blocked triangular solves, row-major (dense_lu.cu):
//   trsm_lower<T, UNIT>:  X := L^-1 X, L the w x w lower block at (r, r) of A
//   trsm_upper<T, TRANS>: X := U^-1 X, U the upper block at (r, r) of A, or
//                         with TRANS X := L^-T X reading the lower block
// X = rows [r, r+w) x cols [c0, c1) of B.
template <typename T, bool UNIT>
int trsm_lower(const GemmSub &gs, const T *A, int64_t lda, int r, int w, T *B, int64_t ldb, int c0,
               int c1);
template <typename T, bool TRANS>
int trsm_upper(const GemmSub &gs, const T *A, int64_t lda, int r, int w, T *B, int64_t ldb, int c0,
               int c1);

// Recursive LU with partial pivoting of the n x n row-major A (dense_lu.cu),
// trailing updates through `gs`.  ipiv/info as nmx_getrf_*.  `tournament`
// (FP32 only) picks each leaf's pivots by tournament pivoting instead: a
// stable LU with other pivots than numax's, for the factorization that
// iterative refinement corrects.
template <typename T>
int getrf_run(nmx_ctx ctx, const GemmSub &gs, int64_t n, T *A, int64_t lda, int32_t *ipiv,
              int32_t *info, bool tournament = false);

// The tallest panel the tournament-pivoting leaf takes (dense_lu.cu).
int64_t tournament_max_rows();

// Rows 0..n-1 of B (ncols columns) interchanged in order as ipiv says
// (numax's laswp on a right-hand-side block; dense_lu.cu).
template <typename T>
void laswp_rows(cudaStream_t st, T *B, int64_t ldb, int n, int ncols, const int32_t *ipiv);

// Recursive lower Cholesky of the n x n row-major A in place (dense_potrf.cu),
// numax's potrf_diag rule at the leaves, updates through `gs` (its precision
// sends the FP32 SYRK / triangular-solve products to the tensor cores).  The
// strict upper triangle is scratch; *info (device) gets the first failing
// pivot.
template <typename T>
int potrf_run(const GemmSub &gs, int64_t n, T *A, int64_t lda, int32_t *info);

}  // namespace nmx
