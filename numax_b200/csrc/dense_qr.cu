// Blocked Householder QR (m >= n) and the thin Q (sm_100a), row-major.
//
// numax's qr_factor (numax/linalg/qr.mojo:615-743) factors each 16-column
// panel with a single-CTA geqr2_panel (numax/linalg/panel.mojo:1975-2073) --
// the documented cap for tall matrices -- then applies the block reflector
// to the trailing columns with three matmuls, C -= V (T^T (V^T C))
// (numax/linalg/qr.mojo:123-327), T built by larft_panel
// (numax/linalg/panel.mojo:2076-2169).
//
// Here the panel is a cooperative kernel over every SM: each CTA keeps its
// share of the panel's rows in shared memory; per column, one grid barrier
// reduces the column norm (every CTA sums the same partials in the same
// order, so all agree on beta and tau), a second reduces the dot products
// with the remaining panel columns.  The same pass accumulates the panel's
// Gram matrix V^T V for T and writes V densely (unit diagonal, zeros above)
// for the GEMMs.  numax's reflector convention is kept exactly:
// beta = -sign(alpha) ||x|| (alpha <= 0 gives +||x||), tau = (beta-alpha)/beta,
// v = x / (alpha - beta), tau = 0 when the sub-column is exactly zero.
#include <algorithm>

#include "dense_common.cuh"

namespace nmx {

constexpr int kQrW = 16;  // panel width (numax's default block)
constexpr int kQrThreads = 256;

template <typename T>
struct QrScratch {
    T *part;        // [2][G][kQrW + 1] per-CTA partial sums (double-buffered)
    T *alpha;       // [2] a[col][col] published by its owner
    T *gram_part;   // [G][kQrW * kQrW]
    unsigned *bar;
    int *err;
};

template <typename T>
__device__ __forceinline__ T block_sum(T v, T *red) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    __syncthreads();
    if (lane == 0) red[warp] = v;
    __syncthreads();
    T t = T(0);
    for (int w = 0; w < kQrThreads / 32; ++w) t += red[w];
    return t;
}

// Factor panel columns [k, k+w) over rows [k, m) in place; Vd receives V
// (rows [k, m) x w, row-major ld kQrW) and tau[k..k+w) the scales.
template <typename T>
__global__ void __launch_bounds__(kQrThreads)
    geqr2_coop_kernel(T *A, int64_t lda, int m, int k, int w, int rows_per_cta, T *tau, T *Vd,
                      QrScratch<T> sc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int ldl = kQrW + 1;
    T *loc = reinterpret_cast<T *>(smem_raw);
    __shared__ T red[kQrThreads / 32];
    __shared__ T s_fac[kQrW];
    __shared__ int s_flag;
    const int G = gridDim.x, cta = blockIdx.x, tid = threadIdx.x;
    const int r0 = k + cta * rows_per_cta;
    const int nloc = max(0, min(rows_per_cta, m - r0));
    for (int e = tid; e < nloc * w; e += kQrThreads) {
        int r = e / w, j = e - r * w;
        loc[r * ldl + j] = A[(int64_t)(r0 + r) * lda + k + j];
    }
    __syncthreads();
    unsigned gen = 0;
    for (int j = 0; j < w; ++j) {
        const int col = k + j;
        const int slot = j & 1;
        const bool own_col = col >= r0 && col < r0 + nloc;
        // ||x||^2 over rows strictly below the diagonal.
        T partial = T(0);
        for (int r = tid; r < nloc; r += kQrThreads)
            if (r0 + r > col) {
                T v = loc[r * ldl + j];
                partial += v * v;
            }
        partial = block_sum(partial, red);
        if (tid == 0) sc.part[((size_t)slot * G + cta) * (kQrW + 1)] = partial;
        if (own_col && tid == 0) sc.alpha[slot] = loc[(col - r0) * ldl + j];
        if (!grid_barrier(sc.bar, gen++, (unsigned)G, sc.err, &s_flag)) return;
        T below = T(0);
        for (int g = 0; g < G; ++g) below += __ldcg(&sc.part[((size_t)slot * G + g) * (kQrW + 1)]);
        const T alpha = __ldcg(&sc.alpha[slot]);
        T this_tau = T(0), scale = T(0), beta = alpha;
        const bool reflect = below != T(0);
        if (reflect) {
            beta = sqrt(alpha * alpha + below);
            if (alpha > T(0)) beta = -beta;
            this_tau = (beta - alpha) / beta;
            scale = T(1) / (alpha - beta);
            for (int r = tid; r < nloc; r += kQrThreads)
                if (r0 + r > col) loc[r * ldl + j] *= scale;
            if (own_col && tid == 0) loc[(col - r0) * ldl + j] = beta;
        }
        if (cta == 0 && tid == 0) tau[col] = this_tau;
        __syncthreads();
        if (!reflect || j + 1 == w) continue;
        // dot_c = a[col][c] + sum_{r > col} v_r a[r][c] for the remaining panel columns.
        for (int c = j + 1; c < w; ++c) {
            T d = T(0);
            for (int r = tid; r < nloc; r += kQrThreads) {
                const int gr = r0 + r;
                if (gr > col) d += loc[r * ldl + j] * loc[r * ldl + c];
                else if (gr == col) d += loc[r * ldl + c];
            }
            d = block_sum(d, red);
            if (tid == 0) sc.part[((size_t)slot * G + cta) * (kQrW + 1) + c] = d;
        }
        if (!grid_barrier(sc.bar, gen++, (unsigned)G, sc.err, &s_flag)) return;
        if (tid < w && tid > j) {
            T d = T(0);
            for (int g = 0; g < G; ++g) d += __ldcg(&sc.part[((size_t)slot * G + g) * (kQrW + 1) + tid]);
            s_fac[tid] = this_tau * d;
        }
        __syncthreads();
        for (int r = tid; r < nloc; r += kQrThreads) {
            const int gr = r0 + r;
            if (gr > col) {
                const T v = loc[r * ldl + j];
                for (int c = j + 1; c < w; ++c) loc[r * ldl + c] -= s_fac[c] * v;
            } else if (gr == col) {
                for (int c = j + 1; c < w; ++c) loc[r * ldl + c] -= s_fac[c];
            }
        }
        __syncthreads();
    }
    // Write the factored panel back and the dense V (unit diagonal, zeros above).
    for (int e = tid; e < nloc * w; e += kQrThreads) {
        const int r = e / w, j = e - r * w, gr = r0 + r;
        const T v = loc[r * ldl + j];
        A[(int64_t)gr * lda + k + j] = v;
        const int rel = gr - k;
        Vd[(int64_t)rel * kQrW + j] = rel > j ? v : (rel == j ? T(1) : T(0));
    }
    // Partial Gram matrix V^T V of this CTA's rows.
    __syncthreads();
    for (int e = tid; e < w * w; e += kQrThreads) {
        const int p = e / w, q = e - p * w;
        T s = T(0);
        for (int r = 0; r < nloc; ++r) {
            const int rel = r0 + r - k;
            const T vp = rel > p ? loc[r * ldl + p] : (rel == p ? T(1) : T(0));
            const T vq = rel > q ? loc[r * ldl + q] : (rel == q ? T(1) : T(0));
            s += vp * vq;
        }
        sc.gram_part[(size_t)cta * kQrW * kQrW + p * kQrW + q] = s;
    }
}

// T (or T^T when `transposed`) of the block reflector from the Gram matrix
// and taus, numax's larft (numax/linalg/panel.mojo:2076-2169): one thread.
template <typename T>
__global__ void larft_kernel(const T *gram_part, int G, const T *tau, int k, int w, T *Tm,
                             int transposed) {
    __shared__ T g[kQrW][kQrW];
    __shared__ T t[kQrW][kQrW];
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
        const int p = e / w, q = e - p * w;
        T s = T(0);
        for (int c = 0; c < G; ++c) s += gram_part[(size_t)c * kQrW * kQrW + p * kQrW + q];
        g[p][q] = s;
        t[p][q] = T(0);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        t[0][0] = tau[k];
        for (int i = 1; i < w; ++i) {
            const T ti = tau[k + i];
            for (int p = 0; p < i; ++p) t[p][i] = -ti * g[p][i];
            for (int q = 0; q < i; ++q) {
                T s = T(0);
                for (int r = q; r < i; ++r) s += t[q][r] * t[r][i];
                t[q][i] = s;
            }
            t[i][i] = ti;
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kQrW * kQrW; e += blockDim.x) {
        const int p = e / kQrW, q = e - p * kQrW;
        T v = (p < w && q < w) ? (transposed ? t[q][p] : t[p][q]) : T(0);
        Tm[p * kQrW + q] = v;
    }
}

// W = V^T C over the rows of a tall panel, split by rows: CTA (g, b) forms
// the partial product of row chunk g with columns [256 b, 256 b + 256) of C
// -- one thread per column, kQrW accumulators, V's rows staged through
// shared memory -- and leaves it at part[g] (kQrW x nc).  Reads C once.
constexpr int kVtcRows = 64;
constexpr int kVtcMaxChunks = 512;
template <typename T>
__global__ void __launch_bounds__(256) vtc_partial_kernel(const T *V, const T *C, int64_t ldc,
                                                          int mk, int nc, int rows_per, T *part) {
    __shared__ T vs[kVtcRows][kQrW];
    const int g = blockIdx.x;
    const int c = blockIdx.y * 256 + threadIdx.x;
    const int r0 = g * rows_per, r1 = min(mk, r0 + rows_per);
    T acc[kQrW];
#pragma unroll
    for (int j = 0; j < kQrW; ++j) acc[j] = T(0);
    for (int rb = r0; rb < r1; rb += kVtcRows) {
        const int nr = min(kVtcRows, r1 - rb);
        __syncthreads();
        for (int e = threadIdx.x; e < kVtcRows * kQrW; e += 256) {
            const int i = e / kQrW, j = e - i * kQrW;
            vs[i][j] = i < nr ? V[(int64_t)(rb + i) * kQrW + j] : T(0);
        }
        __syncthreads();
        if (c < nc) {
            const T *col = C + (int64_t)rb * ldc + c;
#pragma unroll 4
            for (int i = 0; i < nr; ++i) {
                const T x = col[(int64_t)i * ldc];
#pragma unroll
                for (int j = 0; j < kQrW; ++j) acc[j] += vs[i][j] * x;
            }
        }
    }
    if (c < nc)
#pragma unroll
        for (int j = 0; j < kQrW; ++j) part[((int64_t)g * kQrW + j) * nc + c] = acc[j];
}

// W = sum over the G partials (in chunk order, so every run sums alike), then
// Y = Tm W (kQrW x kQrW times kQrW x nc), or Y = W when Tm is null.  A CTA per
// 16 columns, thread (j, c).
template <typename T>
__global__ void __launch_bounds__(kQrW * 16) vtc_reduce_kernel(const T *part, int G, int nc,
                                                              const T *Tm, T *Y) {
    __shared__ T w[kQrW][17];
    const int j = threadIdx.x / 16, cc = threadIdx.x % 16, c = blockIdx.x * 16 + cc;
    T s = T(0);
    if (c < nc) {
#pragma unroll 8
        for (int g = 0; g < G; ++g) s += part[((int64_t)g * kQrW + j) * nc + c];
    }
    w[j][cc] = s;
    __syncthreads();
    if (c >= nc) return;
    if (Tm) {
        T y = T(0);
#pragma unroll
        for (int p = 0; p < kQrW; ++p) y += Tm[j * kQrW + p] * w[p][cc];
        Y[(int64_t)j * nc + c] = y;
    } else {
        Y[(int64_t)j * nc + c] = s;
    }
}

template <typename T>
struct QrRun {
    nmx_ctx ctx;
    cudaStream_t st;
    int m;
    T *Vd, *Tm, *Yk;  // V (m x 16), T (16 x 16), Y (16 x n)
    T *part;          // kVtcMaxChunks x 16 x n partial products
    QrScratch<T> sc;
};

// Y = Tm V^T C (Tm null: Y = V^T C) for the mk x nc block C.
template <typename T>
static int vtc(QrRun<T> &R, int mk, const T *C, int64_t ldc, int nc, const T *Tm, T *Y) {
    const int cb = (int)ceil_div(nc, 256);
    int G = (int)std::min<int64_t>({ceil_div(mk, 256), (int64_t)kVtcMaxChunks,
                                    std::max<int64_t>(1, 4 * (int64_t)R.ctx->sm_count / cb)});
    G = std::max(G, 1);
    const int rows_per = (int)ceil_div(mk, G);
    G = (int)ceil_div(mk, rows_per);
    vtc_partial_kernel<T><<<dim3(G, cb), 256, 0, R.st>>>(R.Vd, C, ldc, mk, nc, rows_per, R.part);
    vtc_reduce_kernel<T><<<(unsigned)ceil_div(nc, 16), kQrW * 16, 0, R.st>>>(R.part, G, nc, Tm, Y);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

// Factor the panel at column k (width w) and record V and T' for it.
template <typename T>
static int qr_panel(QrRun<T> &R, T *A, int64_t lda, T *tau, int k, int w, int transposed) {
    const int mk = R.m - k;
    int G = (int)std::min<int64_t>(R.ctx->sm_count, ceil_div(mk, 64));
    G = std::max(G, 1);
    int rpc = (int)ceil_div(mk, G);
    G = (int)ceil_div(mk, rpc);
    const size_t smem = sizeof(T) * (size_t)rpc * (kQrW + 1);
    if (smem > R.ctx->smem_optin - 1024) {
        set_error("QR panel of %d rows does not fit the cooperative grid", mk);
        return NMX_ERR_UNSUPPORTED;
    }
    NMX_CUDA_TRY(cudaMemsetAsync(R.sc.bar, 0, sizeof(unsigned), R.st));
    NMX_CUDA_TRY(cudaMemsetAsync(R.Vd, 0, sizeof(T) * (size_t)mk * kQrW, R.st));
    void *args[] = {&A, &lda, &R.m, &k, &w, &rpc, &tau, &R.Vd, &R.sc};
    NMX_CUDA_TRY(cudaLaunchCooperativeKernel((void *)geqr2_coop_kernel<T>, dim3(G), dim3(kQrThreads),
                                             args, smem, R.st));
    larft_kernel<T><<<1, 256, 0, R.st>>>(R.sc.gram_part, G, tau, k, w, R.Tm, transposed);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

// C := (I - V T' V^T) C for C = rows [k, m) x cols [c0, c1) of Cm.
template <typename T>
static int apply_reflector(QrRun<T> &R, int k, T *Cm, int64_t ldc, int c0, int c1) {
    const int nc = c1 - c0, mk = R.m - k;
    if (nc <= 0) return 0;
    T *C = Cm + (int64_t)k * ldc + c0;
    // Y = T' (V^T C), then C -= V Y.
    NMX_TRY(vtc<T>(R, mk, C, ldc, nc, R.Tm, R.Yk));
    return gemm_cc<T>(R.st, false, false, mk, nc, kQrW, T(-1), R.Vd, kQrW, R.Yk, nc, T(1), C, ldc);
}

template <typename T>
static int qr_setup(nmx_ctx ctx, cudaStream_t st, int64_t m, int64_t n, QrRun<T> &R) {
    const int G = ctx->sm_count;
    const size_t nn = (size_t)std::max<int64_t>(n, kQrW);
    size_t elems = (size_t)m * kQrW + kQrW * kQrW + (size_t)kQrW * nn +
                   (size_t)kVtcMaxChunks * kQrW * nn + 2 * (size_t)G * (kQrW + 1) + 2 +
                   (size_t)G * kQrW * kQrW + 64;
    void *wsv = nullptr;
    int rc = ctx->ensure_slot(kWsWork, sizeof(T) * elems + 64, &wsv);
    if (rc) return rc;
    T *ws = static_cast<T *>(wsv);
    R.ctx = ctx;
    R.st = st;
    R.m = (int)m;
    R.Vd = ws;
    R.Tm = R.Vd + (size_t)m * kQrW;
    R.Yk = R.Tm + kQrW * kQrW;
    R.part = R.Yk + (size_t)kQrW * nn;
    R.sc.part = R.part + (size_t)kVtcMaxChunks * kQrW * nn;
    R.sc.alpha = R.sc.part + 2 * (size_t)G * (kQrW + 1);
    R.sc.gram_part = R.sc.alpha + 2;
    R.sc.bar = reinterpret_cast<unsigned *>(R.sc.gram_part + (size_t)G * kQrW * kQrW);
    R.sc.err = reinterpret_cast<int *>(R.sc.bar + 1);
    NMX_CUDA_TRY(cudaMemsetAsync(R.sc.err, 0, sizeof(int), st));
    NMX_CUDA_TRY(cudaFuncSetAttribute(geqr2_coop_kernel<T>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(ctx->smem_optin - 1024)));
    return 0;
}

template <typename T>
static int geqrf(nmx_ctx ctx, int64_t m, int64_t n, T *A, int64_t lda, T *tau, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(m >= 0 && m < (int64_t(1) << 31), 2, "m out of range");
    NMX_ARG_CHECK(n >= 0 && n <= m, 3, "need 0 <= n <= m");
    NMX_ARG_CHECK(A != nullptr || n == 0, 4, "A is NULL");
    NMX_ARG_CHECK(lda >= std::max<int64_t>(1, n), 5, "lda < max(1, n)");
    NMX_ARG_CHECK(tau != nullptr || n == 0, 6, "tau is NULL");
    if (n == 0) return 0;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    QrRun<T> R;
    int rc = qr_setup<T>(ctx, st, m, n, R);
    if (rc) return rc;
    for (int k = 0; k < n; k += kQrW) {
        const int w = (int)std::min<int64_t>(kQrW, n - k);
        rc = qr_panel<T>(R, A, lda, tau, k, w, 1);
        if (rc) return rc;
        rc = apply_reflector<T>(R, k, A, lda, k + w, (int)n);
        if (rc) return rc;
    }
    return 0;
}

template <typename T>
__global__ void identity_kernel(T *Q, int64_t ldq, int m, int n) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)m * n) return;
    const int i = (int)(e / n), j = (int)(e - (int64_t)i * n);
    Q[(int64_t)i * ldq + j] = i == j ? T(1) : T(0);
}

// Pack V of the panel at k (read from the factored A) and its T into R.
template <typename T>
__global__ void pack_v_kernel(const T *A, int64_t lda, int m, int k, int w, T *Vd, T *gram_part) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const int64_t mk = m - k;
    if (e >= mk * kQrW) return;
    const int rel = (int)(e / kQrW), j = (int)(e - (int64_t)rel * kQrW);
    T v = T(0);
    if (j < w) v = rel > j ? A[(int64_t)(k + rel) * lda + k + j] : (rel == j ? T(1) : T(0));
    Vd[e] = v;
}

template <typename T>
static int orgqr(nmx_ctx ctx, int64_t m, int64_t n, const T *F, int64_t ldf, const T *tau, T *Q,
                 int64_t ldq, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(m >= 0 && m < (int64_t(1) << 31), 2, "m out of range");
    NMX_ARG_CHECK(n >= 0 && n <= m, 3, "need 0 <= n <= m");
    NMX_ARG_CHECK(F != nullptr || n == 0, 4, "F is NULL");
    NMX_ARG_CHECK(ldf >= std::max<int64_t>(1, n), 5, "ldf < max(1, n)");
    NMX_ARG_CHECK(tau != nullptr || n == 0, 6, "tau is NULL");
    NMX_ARG_CHECK(Q != nullptr || n == 0, 7, "Q is NULL");
    NMX_ARG_CHECK(ldq >= std::max<int64_t>(1, n), 8, "ldq < max(1, n)");
    if (n == 0) return 0;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    QrRun<T> R;
    int rc = qr_setup<T>(ctx, st, m, n, R);
    if (rc) return rc;
    identity_kernel<T><<<(unsigned)ceil_div(m * n, 256), 256, 0, st>>>(Q, ldq, (int)m, (int)n);
    NMX_CUDA_TRY(cudaGetLastError());
    const int steps = (int)ceil_div(n, kQrW);
    for (int s = 0; s < steps; ++s) {
        const int k = (steps - 1 - s) * kQrW;
        const int w = (int)std::min<int64_t>(kQrW, n - k);
        const int64_t mk = m - k;
        pack_v_kernel<T><<<(unsigned)ceil_div(mk * kQrW, 256), 256, 0, st>>>(F, ldf, (int)m, k, w,
                                                                             R.Vd, nullptr);
        NMX_CUDA_TRY(cudaGetLastError());
        // Gram matrix of V for T (one partial), then T.
        NMX_TRY(vtc<T>(R, (int)mk, R.Vd, kQrW, kQrW, nullptr, R.sc.gram_part));
        larft_kernel<T><<<1, 256, 0, st>>>(R.sc.gram_part, 1, tau, k, w, R.Tm, 0);
        NMX_CUDA_TRY(cudaGetLastError());
        rc = apply_reflector<T>(R, k, Q, ldq, k, (int)n);
        if (rc) return rc;
    }
    return 0;
}

// B := Q^T B for the m x nrhs block B (ldb): numax's QR.apply_q_transpose
// (numax/linalg/qr.mojo:470-530) -- the reflectors in factorization order,
// each panel through its block reflector (T^T), Q never formed.
template <typename T>
static int ormqr(nmx_ctx ctx, int64_t m, int64_t n, const T *F, int64_t ldf, const T *tau, T *B,
                 int64_t ldb, int64_t nrhs, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(m >= 0 && m < (int64_t(1) << 31), 2, "m out of range");
    NMX_ARG_CHECK(n >= 0 && n <= m, 3, "need 0 <= n <= m");
    NMX_ARG_CHECK(F != nullptr || n == 0, 4, "F is NULL");
    NMX_ARG_CHECK(ldf >= std::max<int64_t>(1, n), 5, "ldf < max(1, n)");
    NMX_ARG_CHECK(tau != nullptr || n == 0, 6, "tau is NULL");
    NMX_ARG_CHECK(B != nullptr || nrhs == 0 || m == 0, 7, "B is NULL");
    NMX_ARG_CHECK(ldb >= std::max<int64_t>(1, nrhs), 8, "ldb < max(1, nrhs)");
    NMX_ARG_CHECK(nrhs >= 0, 9, "nrhs < 0");
    if (n == 0 || nrhs == 0) return 0;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    QrRun<T> R;
    NMX_TRY(qr_setup<T>(ctx, st, m, std::max<int64_t>(n, nrhs), R));
    for (int k = 0; k < n; k += kQrW) {
        const int w = (int)std::min<int64_t>(kQrW, n - k);
        const int64_t mk = m - k;
        pack_v_kernel<T><<<(unsigned)ceil_div(mk * kQrW, 256), 256, 0, st>>>(F, ldf, (int)m, k, w,
                                                                             R.Vd, nullptr);
        NMX_CUDA_TRY(cudaGetLastError());
        NMX_TRY(vtc<T>(R, (int)mk, R.Vd, kQrW, kQrW, nullptr, R.sc.gram_part));
        larft_kernel<T><<<1, 256, 0, st>>>(R.sc.gram_part, 1, tau, k, w, R.Tm, 1);
        NMX_CUDA_TRY(cudaGetLastError());
        NMX_TRY(apply_reflector<T>(R, k, B, ldb, 0, (int)nrhs));
    }
    return 0;
}

// x = argmin ||A x - b||: numax's QR.solve (numax/linalg/qr.mojo:532-612),
// Q^T b (into b's copy `work`, m values) then the back substitution with R.
template <typename T>
static int qr_solve(nmx_ctx ctx, int64_t m, int64_t n, const T *F, int64_t ldf, const T *tau,
                    const T *b, T *x, T *work, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(m >= 0 && m < (int64_t(1) << 31), 2, "m out of range");
    NMX_ARG_CHECK(n >= 0 && n <= m, 3, "need 0 <= n <= m");
    NMX_ARG_CHECK(F != nullptr || n == 0, 4, "F is NULL");
    NMX_ARG_CHECK(ldf >= std::max<int64_t>(1, n), 5, "ldf < max(1, n)");
    NMX_ARG_CHECK(tau != nullptr || n == 0, 6, "tau is NULL");
    NMX_ARG_CHECK(b != nullptr || m == 0, 7, "b is NULL");
    NMX_ARG_CHECK(x != nullptr || n == 0, 8, "x is NULL");
    NMX_ARG_CHECK(work != nullptr || m == 0, 9, "work is NULL");
    if (n == 0) return 0;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    NMX_CUDA_TRY(cudaMemcpyAsync(work, b, sizeof(T) * (size_t)m, cudaMemcpyDeviceToDevice, st));
    NMX_TRY(ormqr<T>(ctx, m, n, F, ldf, tau, work, 1, 1, stream));
    NMX_CUDA_TRY(cudaMemcpyAsync(x, work, sizeof(T) * (size_t)n, cudaMemcpyDeviceToDevice, st));
    GemmSub gs;
    gs.st = st;
    return trsm_upper<T, false>(gs, F, ldf, 0, (int)n, x, 1, 0, 1);
}

}  // namespace nmx

extern "C" {

NMX_API int nmx_ormqr_f32(nmx_ctx ctx, int64_t m, int64_t n, const float *F, int64_t ldf,
                          const float *tau, float *B, int64_t ldb, int64_t nrhs, void *stream) {
    return nmx::ormqr<float>(ctx, m, n, F, ldf, tau, B, ldb, nrhs, stream);
}
NMX_API int nmx_ormqr_f64(nmx_ctx ctx, int64_t m, int64_t n, const double *F, int64_t ldf,
                          const double *tau, double *B, int64_t ldb, int64_t nrhs, void *stream) {
    return nmx::ormqr<double>(ctx, m, n, F, ldf, tau, B, ldb, nrhs, stream);
}
NMX_API int nmx_qr_solve_f32(nmx_ctx ctx, int64_t m, int64_t n, const float *F, int64_t ldf,
                             const float *tau, const float *b, float *x, float *work,
                             void *stream) {
    return nmx::qr_solve<float>(ctx, m, n, F, ldf, tau, b, x, work, stream);
}
NMX_API int nmx_qr_solve_f64(nmx_ctx ctx, int64_t m, int64_t n, const double *F, int64_t ldf,
                             const double *tau, const double *b, double *x, double *work,
                             void *stream) {
    return nmx::qr_solve<double>(ctx, m, n, F, ldf, tau, b, x, work, stream);
}

NMX_API int nmx_geqrf_f32(nmx_ctx ctx, int64_t m, int64_t n, float *A, int64_t lda, float *tau,
                          void *stream) {
    return nmx::geqrf<float>(ctx, m, n, A, lda, tau, stream);
}
NMX_API int nmx_geqrf_f64(nmx_ctx ctx, int64_t m, int64_t n, double *A, int64_t lda, double *tau,
                          void *stream) {
    return nmx::geqrf<double>(ctx, m, n, A, lda, tau, stream);
}
NMX_API int nmx_orgqr_f32(nmx_ctx ctx, int64_t m, int64_t n, const float *F, int64_t ldf,
                          const float *tau, float *Q, int64_t ldq, void *stream) {
    return nmx::orgqr<float>(ctx, m, n, F, ldf, tau, Q, ldq, stream);
}
NMX_API int nmx_orgqr_f64(nmx_ctx ctx, int64_t m, int64_t n, const double *F, int64_t ldf,
                          const double *tau, double *Q, int64_t ldq, void *stream) {
    return nmx::orgqr<double>(ctx, m, n, F, ldf, tau, Q, ldq, stream);
}

}  // extern "C"
