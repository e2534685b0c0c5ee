// Building blocks shared by the dense factorizations (LU, Cholesky, QR):
// the cooperative grid barrier with a bounded wait, the trailing-update GEMM
// dispatch, row interchanges and small triangular solves.  Row-major storage
// with a leading dimension throughout, as numax's Tensor tiles are.
#pragma once

#include <cublas_v2.h>

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

// Blocked triangular solves, row-major (dense_lu.cu):
//   trsm_lower<T, UNIT>:  X := L^-1 X, L the w x w lower block at (r, r) of A
//   trsm_upper<T, TRANS>: X := U^-1 X, U the upper block at (r, r) of A, or
//                         with TRANS X := L^-T X reading the lower block
// X = rows [r, r+w) x cols [c0, c1) of B.
template <typename T, bool UNIT>
int trsm_lower(nmx_ctx ctx, cublasHandle_t h, cudaStream_t st, const T *A, int64_t lda, int r,
               int w, T *B, int64_t ldb, int c0, int c1);
template <typename T, bool TRANS>
int trsm_upper(nmx_ctx ctx, cublasHandle_t h, cudaStream_t st, const T *A, int64_t lda, int r,
               int w, T *B, int64_t ldb, int c0, int c1);

}  // namespace nmx
