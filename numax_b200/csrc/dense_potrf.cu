// Dense Cholesky and cholesky_solve (sm_100a), row-major, lower.
//
// numax's cholesky (numax/linalg/cholesky.mojo:59-396) is right-looking and
// blocked (block 32 on a device): potrf_diag on the diagonal block
// (numax/linalg/panel.mojo:216-286), trsm_right_lower_t on the panel below it
// (numax/linalg/panel.mojo:2316-2408), and the symmetric trailing update in
// MAX's matmul.  Here the same three steps run recursively over halves, so
// the trailing updates are few large SYRK/GEMM calls:
//
//   potrf(A11); L21 := A21 L11^-T; A22 -= L21 L21^T; potrf(A22)
//
// with 32-column leaves factored by one warp in registers.  The leaf keeps
// numax's rule: a pivot d <= 0 is recorded in info (first one, 1-based) and
// floored to 1e-30 so the factorization continues and stays finite.  Only
// the lower triangle is read; the upper triangle is zeroed at the end, as
// numax's `tril` does (numax/linalg/cholesky.mojo:396).
#include <algorithm>

#include "dense_common.cuh"

namespace nmx {

constexpr int kCholLeaf = 32;

// One warp: Cholesky of the w x w (w <= 32) diagonal block at (c, c).
template <typename T>
__global__ void potrf_leaf_kernel(T *A, int64_t lda, int c, int w, int32_t *info) {
    const int lane = threadIdx.x;
    T a[kCholLeaf];
    T *row = A + (int64_t)(c + lane) * lda + c;
#pragma unroll
    for (int j = 0; j < kCholLeaf; ++j) a[j] = (lane < w && j <= lane) ? row[j] : T(0);
    int first_bad = 0;
#pragma unroll
    for (int j = 0; j < kCholLeaf; ++j) {
        if (j < w) {
            T d = __shfl_sync(0xffffffffu, a[j], j);
            if (d <= T(0)) {
                if (first_bad == 0) first_bad = c + j + 1;
                d = pivot_floor<T>::value;
            }
            // 1/l_jj once per column: the column scales by a product
            // instead of a division on every lane (the pivot chain is
            // d -> rsqrt -> scale -> update).
            const T inv = rsqrt(d);
            if (lane == j) a[j] = d * inv;
            if (lane > j) a[j] = a[j] * inv;
            const T lij = a[j];
#pragma unroll
            for (int cc = j + 1; cc < kCholLeaf; ++cc) {
                const T lcj = __shfl_sync(0xffffffffu, lij, cc);
                if (lane > j && cc <= lane) a[cc] -= lij * lcj;
            }
        }
    }
    if (lane < w) {
#pragma unroll
        for (int j = 0; j < kCholLeaf; ++j)
            if (j <= lane) row[j] = a[j];
    }
    if (lane == 0 && first_bad && *info == 0) *info = first_bad;
}

// X := X L^-T for X = rows [r0, r1) x cols [c, c+w) of A and L the w x w
// (w <= 32) lower block at (c, c).  One thread per row.
template <typename T>
__global__ void trsm_right_lt_leaf_kernel(T *A, int64_t lda, int c, int w, int r0, int r1) {
    __shared__ T Ls[kCholLeaf][kCholLeaf + 1];
    __shared__ T inv_d[kCholLeaf];
    // The block's copies all in flight (cp.async), then one wait.
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
        int i = e / w, j = e - i * w;
        const unsigned d = (unsigned)__cvta_generic_to_shared(&Ls[i][j]);
        const T *src = &A[(int64_t)(c + i) * lda + c + j];
        if constexpr (sizeof(T) == 8)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
        else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    // Reciprocals of the diagonal once per block, so each row's solve is a
    // chain of multiply-adds without a division per column.
    if (threadIdx.x < w) inv_d[threadIdx.x] = T(1) / Ls[threadIdx.x][threadIdx.x];
    __syncthreads();
    const int r = r0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= r1) return;
    T *row = A + (int64_t)r * lda + c;
    T x[kCholLeaf];
#pragma unroll
    for (int j = 0; j < kCholLeaf; ++j) x[j] = j < w ? row[j] : T(0);
#pragma unroll
    for (int j = 0; j < kCholLeaf; ++j) {
        if (j < w) {
            T acc = T(0);
#pragma unroll
            for (int p = 0; p < kCholLeaf; ++p)
                if (p < j) acc += x[p] * Ls[j][p];
            x[j] = (x[j] - acc) * inv_d[j];
        }
    }
#pragma unroll
    for (int j = 0; j < kCholLeaf; ++j)
        if (j < w) row[j] = x[j];
}

// X := X L^-T in one kernel for w <= 256 (a multiple of 32): a CTA per 32
// rows of X, held in shared memory.  Warp b first inverts the 32 x 32
// diagonal block b of L (lane j forms column j of the inverse by forward
// substitution), then block by block: X_b -= Y_<b L_b,<b^T (a product with
// L's block row staged transposed in shared memory), Y_b = X_b L_bb^-T.
constexpr int kCholTrsmMaxW = 256;
constexpr int kCholTrsmThreads = 256;
template <typename T>
__host__ __device__ constexpr size_t chol_trsm_smem(int w) {
    return sizeof(T) * ((size_t)32 * (w + 1) + (size_t)w * 33 + (size_t)w * 34);
}

template <typename T>
__global__ void __launch_bounds__(kCholTrsmThreads)
    trsm_right_lt_small_kernel(T *A, int64_t lda, int c, int w, int r0, int r1) {
    extern __shared__ __align__(16) unsigned char chol_smem[];
    const int xp = w + 1;
    T *X = reinterpret_cast<T *>(chol_smem);  // [32][w+1] the CTA's rows
    T *Li = X + 32 * xp;                      // [w/32][32][33] inverted diagonal blocks
    T *Lt = Li + w * 33;                      // [w][34] L's block row b, transposed
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = kCholTrsmThreads / 32;
    const int nb = w / 32;
    const int rb = r0 + 32 * blockIdx.x, nr = min(32, r1 - rb);
    // Copies into shared memory go out as cp.async, all in flight at once.
    auto async8 = [](T *dst, const T *src) {
        const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
        if constexpr (sizeof(T) == 8)
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
        else
            asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
    };
    for (int i = warp; i < 32; i += NW)
        for (int q = lane; q < w; q += 32) {
            if (i < nr)
                async8(&X[i * xp + q], &A[(int64_t)(rb + i) * lda + c + q]);
            else
                X[i * xp + q] = T(0);
        }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    if (warp < nb) {
        T *D = Li + warp * 32 * 33;
        const int cb = c + 32 * warp;
        for (int i = 0; i < 32; ++i) D[i * 33 + lane] = A[(int64_t)(cb + i) * lda + cb + lane];
        __syncwarp();
        const T my_rd = T(1) / D[lane * 33 + lane];
        T x[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            T t = T(0);
#pragma unroll
            for (int p = 0; p < i; ++p) t = fma(D[i * 33 + p], x[p], t);
            const T rdi = __shfl_sync(0xffffffffu, my_rd, i);
            x[i] = i == lane ? rdi : (i < lane ? T(0) : -t * rdi);
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 32; ++i) D[i * 33 + lane] = x[i];
    }
    __syncthreads();
    const int i = tid >> 3, q0 = (tid & 7) * 4;  // this thread's row and 4 columns of a block
    for (int b = 0; b < nb; ++b) {
        const int cb = 32 * b;
        // L's rows [cb, cb+32) x columns [0, cb), transposed: Lt[p][q] = L[cb+q][p].
        for (int q = warp; q < 32; q += NW)
            for (int p = lane; p < cb; p += 32) async8(&Lt[p * 34 + q], &A[(int64_t)(c + cb + q) * lda + c + p]);
        asm volatile("cp.async.commit_group;\ncp.async.wait_all;\n" ::: "memory");
        __syncthreads();
        T acc[4] = {T(0), T(0), T(0), T(0)};
        for (int p = 0; p < cb; ++p) {
            const T xv = X[i * xp + p];
            const T *lt = Lt + p * 34 + q0;
#pragma unroll
            for (int k = 0; k < 4; ++k) acc[k] = fma(xv, lt[k], acc[k]);
        }
        T z[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) z[k] = X[i * xp + cb + q0 + k] - acc[k];
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 4; ++k) X[i * xp + cb + q0 + k] = z[k];
        __syncthreads();
        // Y_b = Z_b Dinv^T: y_q = sum_{p <= q} z_p Dinv[q][p].
        const T *D = Li + b * 32 * 33;
        T y[4] = {T(0), T(0), T(0), T(0)};
        for (int p = 0; p < 32; ++p) {
            const T zp = X[i * xp + cb + p];
#pragma unroll
            for (int k = 0; k < 4; ++k) y[k] = fma(zp, D[(q0 + k) * 33 + p], y[k]);
        }
        __syncthreads();
#pragma unroll
        for (int k = 0; k < 4; ++k) X[i * xp + cb + q0 + k] = y[k];
        __syncthreads();
    }
    for (int r = warp; r < nr; r += NW)
        for (int q = lane; q < w; q += 32) A[(int64_t)(rb + r) * lda + c + q] = X[r * xp + q];
}

template <typename T>
__global__ void zero_upper_kernel(T *A, int64_t lda, int n) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * n) return;
    const int i = (int)(e / n), j = (int)(e - (int64_t)i * n);
    if (j > i) A[(int64_t)i * lda + j] = T(0);
}

// X := X L^-T, X = rows [r0, r1) x cols [c, c+w), L the lower block at (c, c).
template <typename T>
static int trsm_right_lt(const GemmSub &gs, T *A, int64_t lda, int c, int w, int r0,
                         int r1) {
    cudaStream_t st = gs.st;
    if (w <= 0 || r1 <= r0) return 0;
    if (w > kCholLeaf && w <= kCholTrsmMaxW && w % 32 == 0) {
        static bool attr_set[64] = {};
        int dev = 0;
        NMX_CUDA_TRY(cudaGetDevice(&dev));
        if (dev < 64 && !attr_set[dev]) {
            NMX_CUDA_TRY(cudaFuncSetAttribute(trsm_right_lt_small_kernel<T>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)chol_trsm_smem<T>(kCholTrsmMaxW)));
            attr_set[dev] = true;
        }
        trsm_right_lt_small_kernel<T><<<(unsigned)ceil_div(r1 - r0, 32), kCholTrsmThreads,
                                        chol_trsm_smem<T>(w), st>>>(A, lda, c, w, r0, r1);
        NMX_CUDA_TRY(cudaGetLastError());
        return 0;
    }
    if (w <= kCholLeaf) {
        const int threads = 128;
        trsm_right_lt_leaf_kernel<T>
            <<<(unsigned)ceil_div(r1 - r0, threads), threads, 0, st>>>(A, lda, c, w, r0, r1);
        NMX_CUDA_TRY(cudaGetLastError());
        return 0;
    }
    const int hw = (w / 2 + kCholLeaf - 1) / kCholLeaf * kCholLeaf;
    int rc = trsm_right_lt<T>(gs, A, lda, c, hw, r0, r1);
    if (rc) return rc;
    // X_b -= X_a L_ba^T, L_ba = rows [c+hw, c+w) x cols [c, c+hw).
    NMX_TRY(gs.sub_bt(r1 - r0, w - hw, hw, A + (int64_t)r0 * lda + c, lda,
                      A + (int64_t)(c + hw) * lda + c, lda, A + (int64_t)r0 * lda + c + hw, lda));
    return trsm_right_lt<T>(gs, A, lda, c + hw, w - hw, r0, r1);
}

template <typename T>
static int potrf_rec(const GemmSub &gs, T *A, int64_t lda, int c, int w, int32_t *info) {
    cudaStream_t st = gs.st;
    if (w <= kCholLeaf) {
        potrf_leaf_kernel<T><<<1, 32, 0, st>>>(A, lda, c, w, info);
        NMX_CUDA_TRY(cudaGetLastError());
        return 0;
    }
    const int hw = (w / 2 + kCholLeaf - 1) / kCholLeaf * kCholLeaf;
    int rc = potrf_rec<T>(gs, A, lda, c, hw, info);
    if (rc) return rc;
    rc = trsm_right_lt<T>(gs, A, lda, c, hw, c + hw, c + w);
    if (rc) return rc;
    // A22 -= L21 L21^T on the lower triangle.
    NMX_TRY(gs.sub_bt(w - hw, w - hw, hw, A + (int64_t)(c + hw) * lda + c, lda,
                      A + (int64_t)(c + hw) * lda + c, lda, A + (int64_t)(c + hw) * lda + c + hw,
                      lda, true));
    return potrf_rec<T>(gs, A, lda, c + hw, w - hw, info);
}

// ---- blocked right-looking driver of the FP64 / FP32 entry points ----------
// Per 64-column block column k: one panel launch factors the diagonal block
// and solves the rows below it, then one lower-triangle SYRK updates the
// trailing matrix.  Every CTA of the panel factors the 64 x 64 diagonal block
// itself (the same code on the same data, so all agree bit for bit) and
// forms its inverse, so no CTA waits for another; CTA b then solves rows
// [k + jb + 64 b, +64) as X = R L_kk^-T = R W^T, and CTA 0 writes L_kk.
constexpr int kCholNb = 64;
constexpr int kCholPanelThreads = 256;

template <typename T>
__host__ __device__ constexpr size_t chol_panel_smem() {
    return sizeof(T) * 3 * (size_t)kCholNb * (kCholNb + 1);
}

template <typename T>
__global__ void __launch_bounds__(kCholPanelThreads)
    chol_panel_kernel(T *A, int64_t lda, int n, int k, int jb, int c0, int32_t *info) {
    extern __shared__ __align__(16) unsigned char cp_smem[];
    constexpr int ld = kCholNb + 1;
    constexpr int NT = kCholPanelThreads;
    T *D = reinterpret_cast<T *>(cp_smem);  // the diagonal block, then L_kk
    T *Wm = D + kCholNb * ld;               // W = L_kk^-1 (lower), zeros above
    T *R = Wm + kCholNb * ld;               // this CTA's rows of the panel
    __shared__ T s_l[kCholNb];
    __shared__ int s_bad;
    const int tid = threadIdx.x;
    const int r0 = k + jb + blockIdx.x * kCholNb, nr = max(0, min(kCholNb, n - r0));
    {
        // The diagonal block's lower triangle and this CTA's rows, all copies
        // in flight (cp.async); the rest of D and W starts at zero, W = I.
        auto async_copy = [](T *dst, const T *src) {
            const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
            if constexpr (sizeof(T) == 8)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
            else
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
        };
        for (int e = tid; e < jb * jb; e += NT) {
            const int i = e / jb, j = e - i * jb;
            if (j <= i)
                async_copy(&D[i * ld + j], &A[(int64_t)(k + i) * lda + k + j]);
            else
                D[i * ld + j] = T(0);
        }
        for (int e = tid; e < nr * jb; e += NT) {
            const int i = e / jb, j = e - i * jb;
            async_copy(&R[i * ld + j], &A[(int64_t)(r0 + i) * lda + k + j]);
        }
        for (int e = tid; e < kCholNb * kCholNb; e += NT) {
            const int i = e / kCholNb, j = e - i * kCholNb;
            Wm[i * ld + j] = (i == j && i < jb) ? T(1) : T(0);
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
    }
    if (tid == 0) s_bad = 0;
    __syncthreads();
    // numax's potrf_diag rule per column: a pivot d <= 0 is recorded (first
    // one, 1-based) and floored; l_jj = d / sqrt(d), l_ij = a_ij / sqrt(d).
    // W = L^-1 is formed alongside by elimination: row j of W is scaled by
    // 1/sqrt(d), then rows i > j lose l_ij times it.
    for (int j = 0; j < jb; ++j) {
        T d = D[j * ld + j];
        if (d <= T(0)) {
            if (tid == 0 && s_bad == 0) s_bad = c0 + k + j + 1;
            d = pivot_floor<T>::value;
        }
        const T inv = rsqrt(d);
        if (tid == 0) s_l[j] = d * inv;
        for (int i = j + 1 + tid; i < jb; i += NT) D[i * ld + j] *= inv;
        for (int c = tid; c <= j; c += NT) Wm[j * ld + c] *= inv;
        __syncthreads();
        // D22 -= l l^T on the lower triangle below column j; W's rows below
        // j lose l_ij times row j.  Four lanes per row.
        for (int i = j + 1 + (tid >> 2); i < jb; i += NT / 4) {
            const T lij = D[i * ld + j];
#pragma unroll 4
            for (int l = j + 1 + (tid & 3); l <= i; l += 4) D[i * ld + l] -= lij * D[l * ld + j];
#pragma unroll 4
            for (int c = tid & 3; c <= j; c += 4) Wm[i * ld + c] -= lij * Wm[j * ld + c];
        }
        __syncthreads();
    }
    for (int j = tid; j < jb; j += NT) D[j * ld + j] = s_l[j];
    __syncthreads();
    if (blockIdx.x == 0) {
        for (int e = tid; e < jb * jb; e += NT) {
            const int i = e / jb, j = e - i * jb;
            if (j <= i) A[(int64_t)(k + i) * lda + k + j] = D[i * ld + j];
        }
        if (tid == 0 && s_bad && *info == 0) *info = s_bad;
    }
    // X = R W^T for this CTA's rows: thread (rows 4 (t / 16) + u, columns
    // 4 (t % 16) + v), W's zeros above the diagonal doing the masking.
    if (nr > 0) {
        const int rb = 4 * (tid / 16), cb = 4 * (tid % 16);
        T acc[4][4];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v) acc[u][v] = T(0);
        for (int l = 0; l < jb; ++l) {
            T rv[4], wv[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) rv[u] = rb + u < nr ? R[(rb + u) * ld + l] : T(0);
#pragma unroll
            for (int v = 0; v < 4; ++v) wv[v] = Wm[(cb + v) * ld + l];
#pragma unroll
            for (int u = 0; u < 4; ++u)
#pragma unroll
                for (int v = 0; v < 4; ++v) acc[u][v] = fma(rv[u], wv[v], acc[u][v]);
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int v = 0; v < 4; ++v)
                if (rb + u < nr && cb + v < jb)
                    A[(int64_t)(r0 + rb + u) * lda + k + cb + v] = acc[u][v];
    }
}

// A holds the n x n block whose first column is column c0 of the whole
// matrix (for `info`).
template <typename T>
static int potrf_blocked(const GemmSub &gs, T *A, int64_t lda, int n, int c0, int32_t *info) {
    static bool attr_set[64][2] = {};
    int dev = 0;
    NMX_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 64 && !attr_set[dev][sizeof(T) == 8]) {
        NMX_CUDA_TRY(cudaFuncSetAttribute(chol_panel_kernel<T>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)chol_panel_smem<T>()));
        attr_set[dev][sizeof(T) == 8] = true;
    }
    for (int k = 0; k < n; k += kCholNb) {
        const int jb = std::min(kCholNb, n - k);
        const int below = n - k - jb;
        const int grid = std::max(1, (int)ceil_div(below, kCholNb));
        chol_panel_kernel<T><<<grid, kCholPanelThreads, chol_panel_smem<T>(), gs.st>>>(A, lda, n, k,
                                                                                     jb, c0, info);
        NMX_CUDA_TRY(cudaGetLastError());
        if (below > 0)
            NMX_TRY(gs.sub_bt(below, below, jb, A + (int64_t)(k + jb) * lda + k, lda,
                              A + (int64_t)(k + jb) * lda + k, lda,
                              A + (int64_t)(k + jb) * lda + k + jb, lda, true));
    }
    return 0;
}

// Recursive halves above kCholBlockedMax columns (a few large SYRK / TRSM
// products), the blocked driver below (short chains of launches).
constexpr int kCholBlockedMax = 4096;

template <typename T>
static int potrf_hybrid(const GemmSub &gs, T *A, int64_t lda, int c, int w, int32_t *info) {
    if (w <= kCholBlockedMax) return potrf_blocked<T>(gs, A + (int64_t)c * lda + c, lda, w, c, info);
    const int hw = (w / 2 + kCholLeaf - 1) / kCholLeaf * kCholLeaf;
    NMX_TRY(potrf_hybrid<T>(gs, A, lda, c, hw, info));
    NMX_TRY(trsm_right_lt<T>(gs, A, lda, c, hw, c + hw, c + w));
    NMX_TRY(gs.sub_bt(w - hw, w - hw, hw, A + (int64_t)(c + hw) * lda + c, lda,
                      A + (int64_t)(c + hw) * lda + c, lda, A + (int64_t)(c + hw) * lda + c + hw,
                      lda, true));
    return potrf_hybrid<T>(gs, A, lda, c + hw, w - hw, info);
}

template <typename T>
static int potrf(nmx_ctx ctx, int64_t n, T *A, int64_t lda, int32_t *info, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(n >= 0 && n <= (1 << 20), 2, "n out of range");
    NMX_ARG_CHECK(A != nullptr || n == 0, 3, "A is NULL");
    NMX_ARG_CHECK(lda >= std::max<int64_t>(1, n), 4, "lda < max(1, n)");
    NMX_ARG_CHECK(info != nullptr, 5, "info is NULL");
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    NMX_CUDA_TRY(cudaMemsetAsync(info, 0, sizeof(int32_t), st));
    if (n == 0) return 0;
    GemmSub gs;
    gs.st = st;
    int rc = potrf_hybrid<T>(gs, A, lda, 0, (int)n, info);
    if (rc) return rc;
    const int threads = 256;
    zero_upper_kernel<T><<<(unsigned)ceil_div(n * n, threads), threads, 0, st>>>(A, lda, (int)n);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

template <typename T>
static int potrs(nmx_ctx ctx, int64_t n, int64_t nrhs, const T *L, int64_t lda, T *B, int64_t ldb,
                 void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(n >= 0, 2, "n < 0");
    NMX_ARG_CHECK(nrhs >= 0, 3, "nrhs < 0");
    NMX_ARG_CHECK(L != nullptr || n == 0, 4, "L is NULL");
    NMX_ARG_CHECK(lda >= std::max<int64_t>(1, n), 5, "lda < max(1, n)");
    NMX_ARG_CHECK(B != nullptr || n == 0 || nrhs == 0, 6, "B is NULL");
    NMX_ARG_CHECK(ldb >= std::max<int64_t>(1, nrhs), 7, "ldb < max(1, nrhs)");
    if (n == 0 || nrhs == 0) return 0;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    GemmSub gs;
    gs.st = st;
    int rc = trsm_lower<T, false>(gs, L, lda, 0, (int)n, B, ldb, 0, (int)nrhs);
    if (rc) return rc;
    return trsm_upper<T, true>(gs, L, lda, 0, (int)n, B, ldb, 0, (int)nrhs);
}

template <typename T>
int potrf_run(const GemmSub &gs, int64_t n, T *A, int64_t lda, int32_t *info) {
    NMX_CUDA_TRY(cudaMemsetAsync(info, 0, sizeof(int32_t), gs.st));
    if (n == 0) return 0;
    return potrf_rec<T>(gs, A, lda, 0, (int)n, info);
}
template int potrf_run<double>(const GemmSub &, int64_t, double *, int64_t, int32_t *);
template int potrf_run<float>(const GemmSub &, int64_t, float *, int64_t, int32_t *);

}  // namespace nmx

extern "C" {

NMX_API int nmx_potrf_f64(nmx_ctx ctx, int64_t n, double *A, int64_t lda, int32_t *info,
                          void *stream) {
    return nmx::potrf<double>(ctx, n, A, lda, info, stream);
}
NMX_API int nmx_potrf_f32(nmx_ctx ctx, int64_t n, float *A, int64_t lda, int32_t *info,
                          void *stream) {
    return nmx::potrf<float>(ctx, n, A, lda, info, stream);
}
NMX_API int nmx_potrs_f64(nmx_ctx ctx, int64_t n, int64_t nrhs, const double *L, int64_t lda,
                          double *B, int64_t ldb, void *stream) {
    return nmx::potrs<double>(ctx, n, nrhs, L, lda, B, ldb, stream);
}
NMX_API int nmx_potrs_f32(nmx_ctx ctx, int64_t n, int64_t nrhs, const float *L, int64_t lda,
                          float *B, int64_t ldb, void *stream) {
    return nmx::potrs<float>(ctx, n, nrhs, L, lda, B, ldb, stream);
}

}  // extern "C"
