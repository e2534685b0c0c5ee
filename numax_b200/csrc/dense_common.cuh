// Building blocks shared by the dense factorizations (LU, Cholesky, QR):
// the cooperative grid barrier with a bounded wait, the trailing-update GEMM
// dispatch, row interchanges and small triangular solves.  Row-major storage
// with a leading dimension throughout, as numax's Tensor tiles are.
#pragma once

#include <cublas_v2.h>

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

// C[m x n] -= A[m x k] * B[k x n], all row-major with leading dimensions.
// Plain FP64/FP32 products go to cuBLAS (column-major: C^T -= B^T A^T).
inline cublasStatus_t gemm_sub(cublasHandle_t h, int64_t m, int64_t n, int64_t k, const double *A,
                               int64_t lda, const double *B, int64_t ldb, double *C, int64_t ldc) {
    if (m <= 0 || n <= 0 || k <= 0) return CUBLAS_STATUS_SUCCESS;
    const double minus = -1.0, one = 1.0;
    return cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, (int)m, (int)k, &minus, B, (int)ldb, A,
                       (int)lda, &one, C, (int)ldc);
}
inline cublasStatus_t gemm_sub(cublasHandle_t h, int64_t m, int64_t n, int64_t k, const float *A,
                               int64_t lda, const float *B, int64_t ldb, float *C, int64_t ldc) {
    if (m <= 0 || n <= 0 || k <= 0) return CUBLAS_STATUS_SUCCESS;
    const float minus = -1.0f, one = 1.0f;
    return cublasSgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, (int)n, (int)m, (int)k, &minus, B, (int)ldb, A,
                       (int)lda, &one, C, (int)ldc);
}

// C[m x n] -= A[m x k] * B[n x k]^T (row-major), the SYRK-shaped update.
inline cublasStatus_t gemm_sub_bt(cublasHandle_t h, int64_t m, int64_t n, int64_t k,
                                  const double *A, int64_t lda, const double *B, int64_t ldb,
                                  double *C, int64_t ldc) {
    if (m <= 0 || n <= 0 || k <= 0) return CUBLAS_STATUS_SUCCESS;
    const double minus = -1.0, one = 1.0;
    return cublasDgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, (int)n, (int)m, (int)k, &minus, B, (int)ldb, A,
                       (int)lda, &one, C, (int)ldc);
}
inline cublasStatus_t gemm_sub_bt(cublasHandle_t h, int64_t m, int64_t n, int64_t k,
                                  const float *A, int64_t lda, const float *B, int64_t ldb,
                                  float *C, int64_t ldc) {
    if (m <= 0 || n <= 0 || k <= 0) return CUBLAS_STATUS_SUCCESS;
    const float minus = -1.0f, one = 1.0f;
    return cublasSgemm(h, CUBLAS_OP_T, CUBLAS_OP_N, (int)n, (int)m, (int)k, &minus, B, (int)ldb, A,
                       (int)lda, &one, C, (int)ldc);
}

// General row-major GEMM: C[m x n] = alpha op(A)[m x k] op(B)[k x n] + beta C,
// op(X) = X or X^T (X stored row-major with its leading dimension).
inline cublasStatus_t gemm_rm(cublasHandle_t h, bool ta, bool tb, int64_t m, int64_t n, int64_t k,
                              double alpha, const double *A, int64_t lda, const double *B,
                              int64_t ldb, double beta, double *C, int64_t ldc) {
    if (m <= 0 || n <= 0) return CUBLAS_STATUS_SUCCESS;
    return cublasDgemm(h, tb ? CUBLAS_OP_T : CUBLAS_OP_N, ta ? CUBLAS_OP_T : CUBLAS_OP_N, (int)n,
                       (int)m, (int)k, &alpha, B, (int)ldb, A, (int)lda, &beta, C, (int)ldc);
}
inline cublasStatus_t gemm_rm(cublasHandle_t h, bool ta, bool tb, int64_t m, int64_t n, int64_t k,
                              float alpha, const float *A, int64_t lda, const float *B, int64_t ldb,
                              float beta, float *C, int64_t ldc) {
    if (m <= 0 || n <= 0) return CUBLAS_STATUS_SUCCESS;
    return cublasSgemm(h, tb ? CUBLAS_OP_T : CUBLAS_OP_N, ta ? CUBLAS_OP_T : CUBLAS_OP_N, (int)n,
                       (int)m, (int)k, &alpha, B, (int)ldb, A, (int)lda, &beta, C, (int)ldc);
}

#define NMX_CUBLAS_TRY(expr)                                                                 \
    do {                                                                                     \
        cublasStatus_t _s = (expr);                                                          \
        if (_s != CUBLAS_STATUS_SUCCESS) {                                                   \
            ::nmx::set_error("%s:%d: %s -> cublas status %d", __FILE__, __LINE__, #expr,     \
                             (int)_s);                                                       \
            return NMX_ERR_CUDA;                                                             \
        }                                                                                    \
    } while (0)

// The context's cuBLAS handle bound to `st` (created on first use).
int ctx_cublas(nmx_ctx ctx, cudaStream_t st, cublasHandle_t *out);
// A second cuBLAS handle bound to `st`, for work concurrent with the first's.
int ctx_cublas_aux(nmx_ctx ctx, cudaStream_t st, cublasHandle_t *out);
// Creates the context's look-ahead streams and events on first use.
int ctx_lookahead_streams(nmx_ctx ctx);


// The trailing-update product of the recursive factorizations and solves:
// C[m x n] -= A[m x k] B[k x n], row-major.  precision 0 keeps the operands'
// own precision (cuBLAS FP64/FP32 GEMM); NMX_PREC_BF16 / NMX_PREC_FP16 (fp32
// data only) round the operands to 16 bits and run the tcgen05 kernel.
struct GemmSub {
    cublasHandle_t h = nullptr;
    cudaStream_t st = nullptr;
    int precision = 0;
    int64_t tc_min = 256;
    void *ws = nullptr;
    size_t ws_bytes = 0;
    int sm_limit = 0;  // > 0: tensor-core updates on at most this many SMs
    int operator()(int64_t m, int64_t n, int64_t k, const double *A, int64_t lda, const double *B,
                   int64_t ldb, double *C, int64_t ldc) const {
        cublasStatus_t s = gemm_sub(h, m, n, k, A, lda, B, ldb, C, ldc);
        if (s != CUBLAS_STATUS_SUCCESS) {
            set_error("cublasDgemm failed (%d)", (int)s);
            return NMX_ERR_CUDA;
        }
        return 0;
    }
    int operator()(int64_t m, int64_t n, int64_t k, const float *A, int64_t lda, const float *B,
                   int64_t ldb, float *C, int64_t ldc) const {
        // Tensor cores for the updates with both inner dimensions >= tc_min;
        // the thin ones near the recursion's leaves stay FP32 (their operand
        // rounding passes and launches would cost more than they save).
        if (precision && n >= tc_min && k >= tc_min)
            return tc_gemm_sub_f32(st, precision, m, n, k, A, lda, B, ldb, C, ldc, ws, ws_bytes,
                                   sm_limit);
        cublasStatus_t s = gemm_sub(h, m, n, k, A, lda, B, ldb, C, ldc);
        if (s != CUBLAS_STATUS_SUCCESS) {
            set_error("cublasSgemm failed (%d)", (int)s);
            return NMX_ERR_CUDA;
        }
        return 0;
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

}  // namespace nmx
