// What numax derives from a finished LU (sm_100a): the determinant and its
// logarithm, the unpacked P, L, U, and the inverse.
//
//   nmx_lu_slogdet_*  numax's LU.det / LU.slogdet (numax/linalg/lu.mojo:382-451):
//                     sign = swap parity x signs of U's diagonal, ln|det| =
//                     sum of ln|u_ii|; (0, -inf) when a u_ii is exactly 0;
//                     det = sign x prod(u_ii).  Computed on the device from
//                     the packed factor and the pivots (one CTA: the
//                     logarithms and the signs reduced in a fixed order), so
//                     only three scalars come back.
//   nmx_lu_unpack_*   numax's lu -> PLU (numax/linalg/lu.mojo:877-975): L (unit
//                     diagonal) and U split from the packed factor, the
//                     interchanges replayed on the identity into perm (one
//                     warp; perm[i] = the row of A that row i of L U came
//                     from), and P[perm[i]][i] = 1.
//   nmx_inverse_*     numax's inverse (numax/linalg/basic.mojo:149-192): one
//                     LU and one solve against the whole identity (n
//                     right-hand sides: the blocked triangular solves with
//                     the library's GEMM between blocks).
#include <algorithm>
#include <cmath>

#include "dense_common.cuh"

namespace nmx {

constexpr int kDetThreads = 1024;

// out[0] = sign, out[1] = ln|det|, out[2] = det (sign x prod, in index order
// like numax's host loop).  One CTA.
template <typename T>
__global__ void __launch_bounds__(kDetThreads)
    lu_slogdet_kernel(const T *LU, int64_t lda, int n, const int32_t *ipiv, T *out) {
    __shared__ double s_log[kDetThreads];
    __shared__ int s_neg[kDetThreads], s_zero[kDetThreads];
    double lg = 0.0;
    int neg = 0, zero = 0;
    for (int i = threadIdx.x; i < n; i += kDetThreads) {
        const T d = LU[(int64_t)i * lda + i];
        zero |= d == T(0);
        neg += (d < T(0)) + (ipiv[i] != i);
        lg += log(fabs((double)d));
    }
    s_log[threadIdx.x] = lg;
    s_neg[threadIdx.x] = neg;
    s_zero[threadIdx.x] = zero;
    __syncthreads();
    for (int o = kDetThreads / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) {
            s_log[threadIdx.x] += s_log[threadIdx.x + o];
            s_neg[threadIdx.x] += s_neg[threadIdx.x + o];
            s_zero[threadIdx.x] |= s_zero[threadIdx.x + o];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (s_zero[0]) {
            out[0] = T(0);
            out[1] = T(-INFINITY);
            out[2] = T(0);
        } else {
            // The determinant as numax forms it: the swap parity times the
            // diagonal, multiplied in index order.
            T p = T(1);
            int swaps = 0;
            for (int i = 0; i < n; ++i) swaps += ipiv[i] != i;
            p = (swaps & 1) ? T(-1) : T(1);
            for (int i = 0; i < n; ++i) p *= LU[(int64_t)i * lda + i];
            out[0] = (s_neg[0] & 1) ? T(-1) : T(1);
            out[1] = (T)s_log[0];
            out[2] = p;
        }
    }
}

// L (unit lower), U (upper) from the packed factor; either may be null.
template <typename T>
__global__ void lu_split_kernel(const T *LU, int64_t lda, int n, T *L, int64_t ldl, T *U,
                                int64_t ldu) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * n) return;
    const int i = (int)(e / n), j = (int)(e - (int64_t)i * n);
    const T v = LU[(int64_t)i * lda + j];
    if (L) L[(int64_t)i * ldl + j] = i > j ? v : (i == j ? T(1) : T(0));
    if (U) U[(int64_t)i * ldu + j] = i > j ? T(0) : v;
}

// perm = the interchanges replayed in order on the identity (one thread:
// the swaps are sequential by definition), then P[perm[c]][c] = 1.
__global__ void lu_perm_kernel(const int32_t *ipiv, int n, int32_t *perm) {
    if (threadIdx.x != 0) return;
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int j = 0; j < n; ++j) {
        const int k = ipiv[j];
        const int32_t held = perm[j];
        perm[j] = perm[k];
        perm[k] = held;
    }
}

template <typename T>
__global__ void lu_perm_matrix_kernel(const int32_t *perm, int n, T *P, int64_t ldp) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * n) return;
    const int r = (int)(e / n), c = (int)(e - (int64_t)r * n);
    P[(int64_t)r * ldp + c] = perm[c] == r ? T(1) : T(0);
}

template <typename T>
__global__ void identity_fill_kernel(T *X, int64_t ldx, int n) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * n) return;
    const int r = (int)(e / n), c = (int)(e - (int64_t)r * n);
    X[(int64_t)r * ldx + c] = r == c ? T(1) : T(0);
}

template <typename T>
__global__ void copy_matrix_kernel(const T *A, int64_t lda, int n, T *W, int64_t ldw) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * n) return;
    const int r = (int)(e / n), c = (int)(e - (int64_t)r * n);
    W[(int64_t)r * ldw + c] = A[(int64_t)r * lda + c];
}

template <typename T>
static int slogdet(nmx_ctx ctx, int64_t n, const T *LU, int64_t lda, const int32_t *ipiv, T *out,
                   void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(n >= 0 && n <= (1 << 20), 2, "n out of range");
    NMX_ARG_CHECK(LU != nullptr || n == 0, 3, "LU is NULL");
    NMX_ARG_CHECK(lda >= std::max<int64_t>(1, n), 4, "lda < max(1, n)");
    NMX_ARG_CHECK(ipiv != nullptr || n == 0, 5, "ipiv is NULL");
    NMX_ARG_CHECK(out != nullptr, 6, "out is NULL");
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    lu_slogdet_kernel<T><<<1, kDetThreads, 0, st>>>(LU, lda, (int)n, ipiv, out);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

template <typename T>
static int unpack(nmx_ctx ctx, int64_t n, const T *LU, int64_t lda, const int32_t *ipiv, T *P,
                  int64_t ldp, T *L, int64_t ldl, T *U, int64_t ldu, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(n >= 0 && n <= (1 << 20), 2, "n out of range");
    NMX_ARG_CHECK(LU != nullptr || n == 0, 3, "LU is NULL");
    NMX_ARG_CHECK(lda >= std::max<int64_t>(1, n), 4, "lda < max(1, n)");
    NMX_ARG_CHECK(ipiv != nullptr || n == 0 || P == nullptr, 5, "ipiv is NULL");
    NMX_ARG_CHECK(P == nullptr || ldp >= std::max<int64_t>(1, n), 7, "ldp < max(1, n)");
    NMX_ARG_CHECK(L == nullptr || ldl >= std::max<int64_t>(1, n), 9, "ldl < max(1, n)");
    NMX_ARG_CHECK(U == nullptr || ldu >= std::max<int64_t>(1, n), 11, "ldu < max(1, n)");
    if (n == 0) return 0;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const int threads = 256;
    const unsigned grid = (unsigned)ceil_div(n * n, threads);
    if (L || U) lu_split_kernel<T><<<grid, threads, 0, st>>>(LU, lda, (int)n, L, ldl, U, ldu);
    if (P) {
        void *pv = nullptr;
        NMX_TRY(ctx->ensure_slot(kWsAux, sizeof(int32_t) * (size_t)n + 256, &pv));
        int32_t *perm = static_cast<int32_t *>(pv);
        lu_perm_kernel<<<1, 32, 0, st>>>(ipiv, (int)n, perm);
        lu_perm_matrix_kernel<T><<<grid, threads, 0, st>>>(perm, (int)n, P, ldp);
    }
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

template <typename T>
static int inverse(nmx_ctx ctx, int64_t n, const T *A, int64_t lda, T *X, int64_t ldx,
                   int32_t *ipiv, int32_t *info, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(n >= 0 && n <= (1 << 17), 2, "n out of range");
    NMX_ARG_CHECK(A != nullptr || n == 0, 3, "A is NULL");
    NMX_ARG_CHECK(lda >= std::max<int64_t>(1, n), 4, "lda < max(1, n)");
    NMX_ARG_CHECK(X != nullptr || n == 0, 5, "X is NULL");
    NMX_ARG_CHECK(ldx >= std::max<int64_t>(1, n), 6, "ldx < max(1, n)");
    NMX_ARG_CHECK(ipiv != nullptr || n == 0, 7, "ipiv is NULL");
    NMX_ARG_CHECK(info != nullptr, 8, "info is NULL");
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (n == 0) {
        NMX_CUDA_TRY(cudaMemsetAsync(info, 0, sizeof(int32_t), st));
        return 0;
    }
    // The factor goes to a workspace copy (numax factors a copy too); X
    // starts as the identity and is solved in place.
    const int64_t ldw = (n + 7) / 8 * 8;
    void *wv = nullptr;
    NMX_TRY(ctx->ensure_slot(kWsAux, sizeof(T) * (size_t)n * ldw + 256, &wv));
    T *W = static_cast<T *>(wv);
    const int threads = 256;
    const unsigned grid = (unsigned)ceil_div(n * n, threads);
    copy_matrix_kernel<T><<<grid, threads, 0, st>>>(A, lda, (int)n, W, ldw);
    identity_fill_kernel<T><<<grid, threads, 0, st>>>(X, ldx, (int)n);
    NMX_CUDA_TRY(cudaGetLastError());
    GemmSub gs;
    gs.st = st;
    NMX_TRY(getrf_run<T>(ctx, gs, n, W, ldw, ipiv, info, false));
    // P^T: the interchanges applied to the identity's rows, then the two
    // triangular solves with n right-hand sides.
    laswp_rows<T>(st, X, ldx, (int)n, (int)n, ipiv);
    NMX_CUDA_TRY(cudaGetLastError());
    NMX_TRY((trsm_lower<T, true>(gs, W, ldw, 0, (int)n, X, ldx, 0, (int)n)));
    return trsm_upper<T, false>(gs, W, ldw, 0, (int)n, X, ldx, 0, (int)n);
}

}  // namespace nmx

extern "C" {

NMX_API int nmx_lu_slogdet_f64(nmx_ctx ctx, int64_t n, const double *LU, int64_t lda,
                               const int32_t *ipiv, double *out, void *stream) {
    return nmx::slogdet<double>(ctx, n, LU, lda, ipiv, out, stream);
}
NMX_API int nmx_lu_slogdet_f32(nmx_ctx ctx, int64_t n, const float *LU, int64_t lda,
                               const int32_t *ipiv, float *out, void *stream) {
    return nmx::slogdet<float>(ctx, n, LU, lda, ipiv, out, stream);
}
NMX_API int nmx_lu_unpack_f64(nmx_ctx ctx, int64_t n, const double *LU, int64_t lda,
                              const int32_t *ipiv, double *P, int64_t ldp, double *L, int64_t ldl,
                              double *U, int64_t ldu, void *stream) {
    return nmx::unpack<double>(ctx, n, LU, lda, ipiv, P, ldp, L, ldl, U, ldu, stream);
}
NMX_API int nmx_lu_unpack_f32(nmx_ctx ctx, int64_t n, const float *LU, int64_t lda,
                              const int32_t *ipiv, float *P, int64_t ldp, float *L, int64_t ldl,
                              float *U, int64_t ldu, void *stream) {
    return nmx::unpack<float>(ctx, n, LU, lda, ipiv, P, ldp, L, ldl, U, ldu, stream);
}
NMX_API int nmx_inverse_f64(nmx_ctx ctx, int64_t n, const double *A, int64_t lda, double *X,
                            int64_t ldx, int32_t *ipiv, int32_t *info, void *stream) {
    return nmx::inverse<double>(ctx, n, A, lda, X, ldx, ipiv, info, stream);
}
NMX_API int nmx_inverse_f32(nmx_ctx ctx, int64_t n, const float *A, int64_t lda, float *X,
                            int64_t ldx, int32_t *ipiv, int32_t *info, void *stream) {
    return nmx::inverse<float>(ctx, n, A, lda, X, ldx, ipiv, info, stream);
}

}  // extern "C"
