// Mixed-precision LU solve with iterative refinement (sm_100a).
//
// Not in numax (its GPU path is FP32-only and has no refinement); the
// north-star addition for the large solve.  A (FP64, row-major) is factored
// once in low precision and the solution is refined in FP64:
//
//   W = (float) R A C        R, C power-of-two row/column scalings (exact)
//   P W = L U                the recursive LU of dense_lu.cu with its trailing
//                            updates on the tensor cores (BF16 or FP16 in,
//                            FP32 accumulate) or FP32 CUDA cores
//   x = 0, r = b
//   repeat: d = C U^-1 L^-1 P R r   (triangular solves read the FP32 factors,
//                                    arithmetic in FP64)
//           x += d; r = b - A x (FP64 GEMV over the original A)
//   until ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= tol
//
// GMRES-IR (Carson & Higham) replaces the correction solve by restarted
// GMRES on the left-preconditioned system (U^-1 L^-1 P R A C) y = U^-1 L^-1 P R r,
// all Krylov arithmetic in FP64 with A applied in FP64, for conditioning
// beyond what plain refinement with 16-bit factors converges on.
//
// The single-right-hand-side triangular solves are one persistent kernel
// each: CTAs take 64-row blocks in order from an atomic counter, stream the
// block's row segments left of the diagonal as the solution blocks they need
// become ready (a release/acquire counter of finished blocks), then solve the
// 64 x 64 diagonal block.  Every wait is bounded.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dense_common.cuh"
#include "gemm_tc.cuh"

namespace nmx {

constexpr int kTrsvRB = 64;
constexpr int kTrsvThreads = 256;
constexpr int kTrsvPitch = kTrsvRB + 4;
constexpr size_t kTrsvSmem = (sizeof(double) + sizeof(float)) * kTrsvRB * kTrsvPitch;
constexpr long long kTrsvSpin = 1ll << 25;

__device__ __forceinline__ int ld_acquire_i32(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_i32(int *p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Inverse of every 64 x 64 diagonal block of the unit-lower (UPPER = false)
// or upper (UPPER = true) triangle of the FP32 factor, in FP64: one CTA per
// block, thread j forms column j of the inverse by substitution.  Computed
// once per factorization; it turns each block's serial substitution in the
// triangular solves into a 64 x 64 matrix-vector product.
template <bool UPPER>
__global__ void __launch_bounds__(kTrsvRB)
    diag_inverse_kernel(const float *F, int64_t ldf, int n, double *Inv) {
    __shared__ double D[kTrsvRB][kTrsvRB + 1];
    const int b = blockIdx.x, r0 = b * kTrsvRB, rows = min(kTrsvRB, n - r0);
    const int j = threadIdx.x;
    for (int i = 0; i < rows; ++i)
        if (j < rows) D[i][j] = (double)F[(int64_t)(r0 + i) * ldf + r0 + j];
    __syncthreads();
    double x[kTrsvRB];
#pragma unroll
    for (int i = 0; i < kTrsvRB; ++i) x[i] = 0.0;
    if (j < rows) {
        if (!UPPER) {
#pragma unroll
            for (int i = 0; i < kTrsvRB; ++i) {
                double s = (i == j) ? 1.0 : 0.0;
#pragma unroll
                for (int p = 0; p < kTrsvRB; ++p)
                    if (p < i) s -= D[i][p] * x[p];
                x[i] = (i < rows) ? s : 0.0;
            }
        } else {
#pragma unroll
            for (int ii = 0; ii < kTrsvRB; ++ii) {
                const int i = kTrsvRB - 1 - ii;
                if (i < rows) {
                    double s = (i == j) ? 1.0 : 0.0;
#pragma unroll
                    for (int p = 0; p < kTrsvRB; ++p)
                        if (p > i && p < rows) s -= D[i][p] * x[p];
                    x[i] = s / D[i][i];
                }
            }
        }
    }
    double *out = Inv + (size_t)b * kTrsvRB * kTrsvRB;
#pragma unroll
    for (int i = 0; i < kTrsvRB; ++i) out[i * kTrsvRB + j] = (j < rows && i < rows) ? x[i] : 0.0;
}

// Solve with the unit-lower (UPPER = false) or upper (UPPER = true) triangle
// of the FP32 factor F (n x n, ldf) in place on the FP64 vector x, using the
// precomputed FP64 inverses Inv of its 64 x 64 diagonal blocks.
// counter[0]: block ticket, counter[1]: blocks finished, counter[2]: error.
//
// A CTA takes 64-row blocks in solve order.  It accumulates the block's row
// segments against the solution blocks finished so far as they appear, all
// but the adjacent one (the block finished just before it); meanwhile the
// F tile against that adjacent block and the block's Inv are copied into
// shared memory asynchronously.  So once the adjacent block is released,
// what remains on the chain from block to block is one 64-value read of x,
// two 64 x 64 products out of shared memory, and the release.
__device__ __forceinline__ void cp_async_4(unsigned dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_16(unsigned dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all_() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <bool UPPER>
__global__ void __launch_bounds__(kTrsvThreads)
    trsv_f32f64_kernel(const float *F, int64_t ldf, int n, const double *Inv, double *x,
                       int *counter) {
    // Dynamic shared memory: Is[64][68] (Inv of this block, FP64) then
    // Ft[64][68] (the F tile against the adjacent block).  Row pitch 68 with
    // thread (i, part) reading columns part + 4m keeps both conflict-free.
    extern __shared__ __align__(16) unsigned char trsv_smem[];
    auto Is = reinterpret_cast<double(*)[kTrsvPitch]>(trsv_smem);
    auto Ft = reinterpret_cast<float(*)[kTrsvPitch]>(trsv_smem + sizeof(double) * kTrsvRB * kTrsvPitch);
    __shared__ double accS[kTrsvRB], xs[kTrsvRB], ys[kTrsvRB];
    __shared__ int s_blk, s_avail;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int NB = (n + kTrsvRB - 1) / kTrsvRB;
    // Column range of the finished blocks with solve-order indices [d0, d1).
    auto cols = [&](int d0, int d1, int &c0, int &c1) {
        if (!UPPER) {
            c0 = d0 * kTrsvRB;
            c1 = min(n, d1 * kTrsvRB);
        } else {
            c0 = (NB - d1) * kTrsvRB;
            c1 = min(n, (NB - d0) * kTrsvRB);
        }
    };
    // Wait (thread 0, bounded) until more than `done` blocks are finished.
    auto wait_for = [&](int done) -> int {
        if (tid == 0) {
            long long spins = 0;
            int avail;
            while ((avail = ld_acquire_i32(&counter[1])) <= done) {
                if (++spins > kTrsvSpin) {
                    atomicExch(&counter[2], 1);
                    avail = -1;
                    break;
                }
                if (spins > 1024) __nanosleep(32);
            }
            s_avail = avail;
        }
        __syncthreads();
        const int avail = s_avail;
        __syncthreads();
        return avail;
    };
    for (;;) {
        if (tid == 0) s_blk = atomicAdd(&counter[0], 1);
        __syncthreads();
        const int ticket = s_blk;
        __syncthreads();
        if (ticket >= NB) return;
        const int b = UPPER ? NB - 1 - ticket : ticket;  // row block
        const int r0 = b * kTrsvRB, rows = min(kTrsvRB, n - r0);
        // Inv of this block -> shared (16-byte chunks; rows are 64 doubles).
        {
            const unsigned is0 = (unsigned)__cvta_generic_to_shared(&Is[0][0]);
            const double *inv = Inv + (size_t)b * kTrsvRB * kTrsvRB;
            for (int e = tid; e < kTrsvRB * kTrsvRB / 2; e += kTrsvThreads) {
                const int i = e >> 5, c = (e & 31) * 2;
                cp_async_16(is0 + (unsigned)(i * kTrsvPitch + c) * 8u, inv + i * kTrsvRB + c);
            }
        }
        // Row segments against all finished blocks but the adjacent one:
        // warp w owns rows 8w..8w+7, lanes stride the columns.
        double acc[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) acc[q] = 0.0;
        int done = 0;
        while (done < ticket - 1) {
            const int avail = wait_for(done);
            if (avail < 0) {
                cp_async_wait_all_();
                return;
            }
            const int nd = min(avail, ticket - 1);
            int c0, c1;
            cols(done, nd, c0, c1);
            // Two columns per lane (float2 / double2 loads: c0 is a multiple
            // of 64, rows are 32-byte aligned, x 16-byte aligned), the 8 rows
            // and 2 iterations in flight: this stream must keep ahead of the
            // chain of blocks, so it needs memory-level parallelism.
            int c = c0 + 2 * lane;
#pragma unroll 2
            for (; c + 1 < c1; c += 64) {
                const double2 xv = __ldcg(reinterpret_cast<const double2 *>(x + c));
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int i = min(8 * warp + q, rows - 1);
                    const float2 f = *reinterpret_cast<const float2 *>(F + (int64_t)(r0 + i) * ldf + c);
                    acc[q] += (double)f.x * xv.x + (double)f.y * xv.y;
                }
            }
            if (c < c1) {  // an odd last column
                const double xv = __ldcg(&x[c]);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int i = min(8 * warp + q, rows - 1);
                    acc[q] += (double)F[(int64_t)(r0 + i) * ldf + c] * xv;
                }
            }
            done = nd;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            double s = acc[q];
            for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
            if (lane == 0) accS[8 * warp + q] = s;
        }
        // The F tile against the adjacent block -> shared, zero outside.
        int a0 = 0, a1 = 0;
        if (ticket > 0) cols(ticket - 1, ticket, a0, a1);
        {
            const unsigned ft0 = (unsigned)__cvta_generic_to_shared(&Ft[0][0]);
            for (int e = tid; e < kTrsvRB * kTrsvRB; e += kTrsvThreads) {
                const int i = e >> 6, c = e & 63;
                if (i < rows && a0 + c < a1)
                    cp_async_4(ft0 + (unsigned)(i * kTrsvPitch + c) * 4u,
                               F + (int64_t)(r0 + i) * ldf + a0 + c);
                else
                    Ft[i][c] = 0.0f;
            }
        }
        if (ticket > 0) {
            const int avail = wait_for(ticket - 1);
            if (avail < 0) {
                cp_async_wait_all_();
                return;
            }
        }
        if (tid < kTrsvRB) xs[tid] = (a0 + tid < a1) ? __ldcg(&x[a0 + tid]) : 0.0;
        cp_async_wait_all_();
        __syncthreads();
        // ys = x_blk - F_row . x: thread (i, part) sums 16 of the tile's columns.
        const int i = tid >> 2, part = tid & 3;
        {
            double s = 0.0;
#pragma unroll
            for (int m = 0; m < 16; ++m) s += (double)Ft[i][part + 4 * m] * xs[part + 4 * m];
            s += __shfl_xor_sync(0xffffffffu, s, 1);
            s += __shfl_xor_sync(0xffffffffu, s, 2);
            if (part == 0) ys[i] = i < rows ? x[r0 + i] - accS[i] - s : 0.0;
        }
        __syncthreads();
        // x_blk = Inv ys.
        {
            double s = 0.0;
#pragma unroll
            for (int m = 0; m < 16; ++m) s += Is[i][part + 4 * m] * ys[part + 4 * m];
            s += __shfl_xor_sync(0xffffffffu, s, 1);
            s += __shfl_xor_sync(0xffffffffu, s, 2);
            if (part == 0 && i < rows) x[r0 + i] = s;
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) st_release_i32(&counter[1], ticket + 1);
    }
}

// r = b - A x (FP64), one warp per row; rmax <- max |r_i| (as ordered bits).
__global__ void residual_kernel(const double *A, int64_t lda, int n, const double *x,
                                const double *b, double *r, unsigned long long *rmax) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double *row = A + (int64_t)warp * lda;
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int c = lane;
    for (; c + 96 < n; c += 128) {
        s0 += row[c] * x[c];
        s1 += row[c + 32] * x[c + 32];
        s2 += row[c + 64] * x[c + 64];
        s3 += row[c + 96] * x[c + 96];
    }
    for (; c < n; c += 32) s0 += row[c] * x[c];
    double s = (s0 + s1) + (s2 + s3);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (lane == 0) {
        const double v = b[warp] - s;
        r[warp] = v;
        atomicMax(rmax, (unsigned long long)__double_as_longlong(fabs(v)));
    }
}

// max_i sum_j |A_ij| (||A||_inf) and optional per-row max |A_ij|.
__global__ void row_norms_kernel(const double *A, int64_t lda, int n, unsigned long long *norm_inf,
                                 double *rowmax) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double *row = A + (int64_t)warp * lda;
    double s = 0.0, m = 0.0;
    for (int c = lane; c < n; c += 32) {
        const double v = fabs(row[c]);
        s += v;
        m = fmax(m, v);
    }
    for (int o = 16; o > 0; o >>= 1) {
        s += __shfl_xor_sync(0xffffffffu, s, o);
        m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    }
    if (lane == 0) {
        atomicMax(norm_inf, (unsigned long long)__double_as_longlong(s));
        if (rowmax) rowmax[warp] = m;
    }
}

__global__ void absmax_kernel(const double *v, int n, unsigned long long *out) {
    double m = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m = fmax(m, fabs(v[i]));
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) atomicMax(out, (unsigned long long)__double_as_longlong(m));
}

// Power of two nearest 1/m (1 for m == 0 or non-finite m).
__device__ __forceinline__ double pow2_inv(double m) {
    if (!(m > 0.0) || !isfinite(m)) return 1.0;
    return exp2(-rint(log2(m)));
}

// Row scales from the row maxima.
__global__ void row_scale_kernel(const double *rowmax, int n, double *rs, int enabled) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) rs[i] = enabled ? pow2_inv(rowmax[i]) : 1.0;
}

// Column maxima of R A: a grid of column tiles x row chunks, each thread a
// column over its chunk's rows (coalesced across the warp, 4 rows in
// flight), combined with an atomic max on the (nonnegative) bit patterns.
constexpr int kColChunks = 64;
__global__ void col_max_kernel(const double *A, int64_t lda, int n, const double *rs,
                               unsigned long long *cmax) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= n) return;
    const int per = (n + kColChunks - 1) / kColChunks;
    const int i0 = blockIdx.y * per, i1 = min(n, i0 + per);
    double m0 = 0.0, m1 = 0.0, m2 = 0.0, m3 = 0.0;
    int i = i0;
    for (; i + 3 < i1; i += 4) {
        m0 = fmax(m0, fabs(A[(int64_t)i * lda + j] * rs[i]));
        m1 = fmax(m1, fabs(A[(int64_t)(i + 1) * lda + j] * rs[i + 1]));
        m2 = fmax(m2, fabs(A[(int64_t)(i + 2) * lda + j] * rs[i + 2]));
        m3 = fmax(m3, fabs(A[(int64_t)(i + 3) * lda + j] * rs[i + 3]));
    }
    for (; i < i1; ++i) m0 = fmax(m0, fabs(A[(int64_t)i * lda + j] * rs[i]));
    const double m = fmax(fmax(m0, m1), fmax(m2, m3));
    atomicMax(&cmax[j], (unsigned long long)__double_as_longlong(m));
}

// Column scales from the column maxima (1 when equilibration is off).
__global__ void col_scale_kernel(const unsigned long long *cmax, int n, double *cs, int enabled) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < n) cs[j] = enabled ? pow2_inv(__longlong_as_double((long long)cmax[j])) : 1.0;
}

// W = (float)(R A C).
__global__ void scale_to_f32_kernel(const double *A, int64_t lda, int n, const double *rs,
                                    const double *cs, float *W, int64_t ldw) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * n) return;
    const int i = (int)(e / n), j = (int)(e - (int64_t)i * n);
    W[(int64_t)i * ldw + j] = (float)(A[(int64_t)i * lda + j] * rs[i] * cs[j]);
}

// v[i] = s[perm[i]] * rs[perm[i]]  (apply P R to a vector).
__global__ void permute_scale_kernel(const double *s, const int *perm, const double *rs, int n,
                                     double *v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = s[perm[i]] * rs[perm[i]];
}

// x += C v  (or x = C v when assign).
__global__ void axpy_scale_kernel(const double *v, const double *cs, int n, double *x, int assign) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] = assign ? cs[i] * v[i] : x[i] + cs[i] * v[i];
}

__global__ void add_kernel(const double *v, int n, double *x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += v[i];
}

__global__ void scale_vec_kernel(const double *v, const double *cs, int n, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = cs[i] * v[i];
}

// ---- host side ----------------------------------------------------------

struct IrRun {
    nmx_ctx ctx;
    cudaStream_t st;
    cublasHandle_t h;
    int n;
    const double *A;
    int64_t lda;
    float *W;
    int64_t ldw;
    int *perm;
    double *rs, *cs, *v, *r, *tmp, *rowmax;
    int *counters;  // 3 per triangular solve
    double *invL, *invU;  // inverses of the 64 x 64 diagonal blocks of L and U
    unsigned long long *norms;  // [0] ||A||_inf, [1] ||r||, [2] ||x||, [3] ||b||, [4] scratch
};

static double bits_to_double(unsigned long long u) {
    double d;
    std::memcpy(&d, &u, sizeof d);
    return d;
}

// v := U^-1 L^-1 v (the FP32 factors in W, arithmetic in FP64).
static int lu_solve_inplace(IrRun &R, double *v) {
    const int NB = (R.n + kTrsvRB - 1) / kTrsvRB;
    const int want = R.ctx->tune_ir_trsv_ctas > 0 ? (int)R.ctx->tune_ir_trsv_ctas
                                                  : 2 * R.ctx->sm_count;
    const int grid = std::max(1, std::min(NB, want));
    static bool attr_set[64] = {};
    if (R.ctx->device < 64 && !attr_set[R.ctx->device]) {
        NMX_CUDA_TRY(cudaFuncSetAttribute(trsv_f32f64_kernel<false>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsvSmem));
        NMX_CUDA_TRY(cudaFuncSetAttribute(trsv_f32f64_kernel<true>,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTrsvSmem));
        attr_set[R.ctx->device] = true;
    }
    NMX_CUDA_TRY(cudaMemsetAsync(R.counters, 0, 6 * sizeof(int), R.st));
    trsv_f32f64_kernel<false><<<grid, kTrsvThreads, kTrsvSmem, R.st>>>(R.W, R.ldw, R.n, R.invL, v,
                                                                       R.counters);
    trsv_f32f64_kernel<true><<<grid, kTrsvThreads, kTrsvSmem, R.st>>>(R.W, R.ldw, R.n, R.invU, v,
                                                                      R.counters + 3);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

// out = C U^-1 L^-1 P R in   (the preconditioned correction of one residual).
static int precond_apply(IrRun &R, const double *in, double *out) {
    const int threads = 256, blocks = (int)ceil_div(R.n, threads);
    permute_scale_kernel<<<blocks, threads, 0, R.st>>>(in, R.perm, R.rs, R.n, R.tmp);
    int rc = lu_solve_inplace(R, R.tmp);
    if (rc) return rc;
    scale_vec_kernel<<<blocks, threads, 0, R.st>>>(R.tmp, R.cs, R.n, out);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

// out = A in (FP64) via the residual kernel with b = 0 (out = -A in).
static int apply_A(IrRun &R, const double *in, double *out, const double *zero) {
    const int threads = 256, blocks = (int)ceil_div((int64_t)R.n * 32, threads);
    residual_kernel<<<blocks, threads, 0, R.st>>>(R.A, R.lda, R.n, in, zero, out, R.norms + 4);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

static int gesv_ir(nmx_ctx ctx, int64_t n64, const double *A, int64_t lda, const double *b,
                   double *x, int mode, double tol, int max_iter, nmx_ir_stats *stats,
                   void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(n64 >= 1 && n64 <= (1 << 17), 2, "n must be in 1..131072");
    NMX_ARG_CHECK(A != nullptr, 3, "A is NULL");
    NMX_ARG_CHECK(lda >= n64, 4, "lda < n");
    NMX_ARG_CHECK(b != nullptr, 5, "b is NULL");
    NMX_ARG_CHECK(x != nullptr, 6, "x is NULL");
    const int prec = mode & 0xF;
    const bool gmres = (mode & NMX_IR_GMRES) != 0;
    NMX_ARG_CHECK(prec == NMX_IR_BF16 || prec == NMX_IR_FP16 || prec == NMX_IR_FP32 ||
                      prec == NMX_IR_BF16X3,
                  7, "mode must be NMX_IR_BF16/FP16/FP32/BF16X3, optionally | NMX_IR_GMRES");
    NMX_ARG_CHECK(tol >= 0.0, 8, "tol < 0");
    NMX_ARG_CHECK(max_iter >= 1 && max_iter <= 10000, 9, "max_iter must be in 1..10000");
    const int n = (int)n64;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    IrRun R;
    R.ctx = ctx;
    R.st = st;
    R.n = n;
    R.A = A;
    R.lda = lda;
    int rc = ctx_cublas(ctx, st, &R.h);
    if (rc) return rc;
    // Workspace: FP32 factor, vectors, 16-bit GEMM operands.
    R.ldw = (n + 7) / 8 * 8;
    void *wv = nullptr;
    rc = ctx->ensure_slot(kWsWork, sizeof(float) * (size_t)n * R.ldw + 256, &wv);
    if (rc) return rc;
    R.W = static_cast<float *>(wv);
    const int restart = 200;
    size_t vec_bytes = sizeof(double) * (size_t)n * 8 + sizeof(int) * (size_t)n * 2 + 4096;
    void *vv = nullptr;
    rc = ctx->ensure_slot(kWsVec, vec_bytes, &vv);
    if (rc) return rc;
    char *vp = static_cast<char *>(vv);
    R.norms = reinterpret_cast<unsigned long long *>(vp);
    R.counters = reinterpret_cast<int *>(vp + 256);
    double *dv = reinterpret_cast<double *>(vp + 1024);
    R.rs = dv;
    R.cs = dv + n;
    R.v = dv + 2 * (size_t)n;
    R.r = dv + 3 * (size_t)n;
    R.tmp = dv + 4 * (size_t)n;
    R.rowmax = dv + 5 * (size_t)n;
    double *zero = dv + 6 * (size_t)n;
    double *aux = dv + 7 * (size_t)n;
    R.perm = reinterpret_cast<int *>(dv + 8 * (size_t)n);
    int32_t *ipiv = R.perm + n;
    int32_t *info_d = reinterpret_cast<int32_t *>(R.counters + 16);
    GemmSub gs;
    gs.h = R.h;
    gs.st = st;
    gs.precision = prec == NMX_IR_FP32    ? 0
                   : prec == NMX_IR_FP16   ? NMX_PREC_FP16
                   : prec == NMX_IR_BF16X3 ? NMX_PREC_BF16X3
                                           : NMX_PREC_BF16;
    if (ctx->tune_ir_tc_min >= 0) gs.tc_min = ctx->tune_ir_tc_min;
    if (gs.precision) {
        const int64_t half = (n / 2 + 31) / 32 * 32;
        gs.ws_bytes = tc_gemm_workspace_bytes(n - half, n - half, half, gs.precision) + 4096;
        rc = ctx->ensure_slot(kWsGemm16, gs.ws_bytes, &gs.ws);
        if (rc) return rc;
    }
    const int threads = 256;
    const int vb = (int)ceil_div(n, threads);
    const int wb = (int)ceil_div((int64_t)n * 32, threads);
    cudaEvent_t e0, e1, e2;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventCreate(&e2);
    NMX_CUDA_TRY(cudaEventRecord(e0, st));
    // ||A||_inf, equilibration (power-of-two scalings; FP16 factors need the range).
    NMX_CUDA_TRY(cudaMemsetAsync(R.norms, 0, 8 * sizeof(unsigned long long), st));
    NMX_CUDA_TRY(cudaMemsetAsync(zero, 0, sizeof(double) * n, st));
    row_norms_kernel<<<wb, threads, 0, st>>>(A, lda, n, R.norms, R.rowmax);
    const int equil = prec == NMX_IR_FP16 ? 1 : 0;
    row_scale_kernel<<<vb, threads, 0, st>>>(R.rowmax, n, R.rs, equil);
    if (equil) {
        // The column maxima go through R.tmp's bits (free until the solve).
        unsigned long long *cmax = reinterpret_cast<unsigned long long *>(R.tmp);
        NMX_CUDA_TRY(cudaMemsetAsync(cmax, 0, sizeof(double) * n, st));
        col_max_kernel<<<dim3(vb, kColChunks), threads, 0, st>>>(A, lda, n, R.rs, cmax);
        col_scale_kernel<<<vb, threads, 0, st>>>(cmax, n, R.cs, 1);
    } else {
        col_scale_kernel<<<vb, threads, 0, st>>>(nullptr, n, R.cs, 0);
    }
    scale_to_f32_kernel<<<(unsigned)ceil_div((int64_t)n * n, threads), threads, 0, st>>>(
        A, lda, n, R.rs, R.cs, R.W, R.ldw);
    NMX_CUDA_TRY(cudaGetLastError());
    rc = getrf_run<float>(ctx, gs, n, R.W, R.ldw, ipiv, info_d, ctx->tune_lu_tournament != 0);
    if (rc) return rc;
    // Inverses of the diagonal blocks of L and U for the triangular solves.
    {
        const int NB = (n + kTrsvRB - 1) / kTrsvRB;
        void *iv = nullptr;
        rc = ctx->ensure_slot(kWsInv, sizeof(double) * (size_t)NB * kTrsvRB * kTrsvRB * 2 + 256,
                              &iv);
        if (rc) return rc;
        R.invL = static_cast<double *>(iv);
        R.invU = R.invL + (size_t)NB * kTrsvRB * kTrsvRB;
        diag_inverse_kernel<false><<<NB, kTrsvRB, 0, st>>>(R.W, R.ldw, n, R.invL);
        diag_inverse_kernel<true><<<NB, kTrsvRB, 0, st>>>(R.W, R.ldw, n, R.invU);
        NMX_CUDA_TRY(cudaGetLastError());
    }
    NMX_CUDA_TRY(cudaEventRecord(e1, st));
    // Pivots -> permutation on the host (the interchanges compose in order).
    std::vector<int32_t> hp(n), perm(n);
    int32_t hinfo = 0;
    NMX_CUDA_TRY(cudaMemcpyAsync(hp.data(), ipiv, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
    NMX_CUDA_TRY(cudaMemcpyAsync(&hinfo, info_d, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    unsigned long long hnorm[8];
    NMX_CUDA_TRY(cudaMemcpyAsync(hnorm, R.norms, sizeof hnorm, cudaMemcpyDeviceToHost, st));
    NMX_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int j = 0; j < n; ++j)
        if (hp[j] != j) std::swap(perm[j], perm[hp[j]]);
    NMX_CUDA_TRY(cudaMemcpyAsync(R.perm, perm.data(), sizeof(int32_t) * n, cudaMemcpyHostToDevice, st));
    const double normA = bits_to_double(hnorm[0]);
    // ||b||_inf
    absmax_kernel<<<std::min(vb, 1024), threads, 0, st>>>(b, n, R.norms + 3);
    // x = 0, r = b
    NMX_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
    NMX_CUDA_TRY(cudaMemcpyAsync(R.r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    int it = 0, inner_total = 0;
    double berr = INFINITY, prev = INFINITY, best_berr = INFINITY;
    int stalled = 0;
    bool use_gmres = gmres;
    std::vector<double> H((size_t)(restart + 1) * restart), cs_g(restart), sn_g(restart),
        gvec(restart + 1), y(restart);
    void *kv = nullptr;
    for (it = 1; it <= max_iter; ++it) {
        if (!use_gmres) {
            rc = precond_apply(R, R.r, R.v);  // d = M^-1 r
            if (rc) return rc;
            add_kernel<<<vb, threads, 0, st>>>(R.v, n, x);
            NMX_CUDA_TRY(cudaGetLastError());
        } else {
            // Restarted GMRES on M^-1 A d = M^-1 r, M^-1 = C U^-1 L^-1 P R.
            rc = ctx->ensure_slot(kWsKrylov, sizeof(double) * ((size_t)n * (restart + 1) + 2 * 64), &kv);
            if (rc) return rc;
            double *Vk = static_cast<double *>(kv);
            double *hdev = Vk + (size_t)n * (restart + 1);
            std::vector<double> hh(restart + 1);
            rc = precond_apply(R, R.r, Vk);  // z0 = M^-1 r
            if (rc) return rc;
            double beta = 0.0;
            NMX_CUBLAS_TRY(cublasDnrm2(R.h, n, Vk, 1, &beta));
            NMX_CUDA_TRY(cudaStreamSynchronize(st));
            if (!(beta > 0.0)) break;
            const double inv = 1.0 / beta;
            NMX_CUBLAS_TRY(cublasDscal(R.h, n, &inv, Vk, 1));
            std::fill(gvec.begin(), gvec.end(), 0.0);
            gvec[0] = beta;
            int k = 0;
            for (; k < restart; ++k) {
                double *vk = Vk + (size_t)k * n, *w = Vk + (size_t)(k + 1) * n;
                rc = apply_A(R, vk, aux, zero);  // aux = -A vk
                if (rc) return rc;
                const double minus = -1.0;
                NMX_CUBLAS_TRY(cublasDscal(R.h, n, &minus, aux, 1));
                rc = precond_apply(R, aux, w);
                if (rc) return rc;
                // Classical Gram-Schmidt, twice (CGS2): h = V^T w, w -= V h.
                const double one = 1.0, zero_d = 0.0, mone = -1.0;
                for (int pass = 0; pass < 2; ++pass) {
                    NMX_CUBLAS_TRY(cublasDgemv(R.h, CUBLAS_OP_T, n, k + 1, &one, Vk, n, w, 1,
                                               &zero_d, hdev, 1));
                    NMX_CUBLAS_TRY(cublasDgemv(R.h, CUBLAS_OP_N, n, k + 1, &mone, Vk, n, hdev, 1,
                                               &one, w, 1));
                    NMX_CUDA_TRY(cudaMemcpyAsync(hh.data(), hdev, sizeof(double) * (k + 1),
                                                 cudaMemcpyDeviceToHost, st));
                    NMX_CUDA_TRY(cudaStreamSynchronize(st));
                    for (int j = 0; j <= k; ++j)
                        H[(size_t)j * restart + k] = (pass == 0 ? 0.0 : H[(size_t)j * restart + k]) + hh[j];
                }
                double hn = 0.0;
                NMX_CUBLAS_TRY(cublasDnrm2(R.h, n, w, 1, &hn));
                NMX_CUDA_TRY(cudaStreamSynchronize(st));
                H[(size_t)(k + 1) * restart + k] = hn;
                if (hn > 0.0) {
                    const double ih = 1.0 / hn;
                    NMX_CUBLAS_TRY(cublasDscal(R.h, n, &ih, w, 1));
                }
                // Givens rotations on column k of H.
                for (int j = 0; j < k; ++j) {
                    const double a = H[(size_t)j * restart + k], bb = H[(size_t)(j + 1) * restart + k];
                    H[(size_t)j * restart + k] = cs_g[j] * a + sn_g[j] * bb;
                    H[(size_t)(j + 1) * restart + k] = -sn_g[j] * a + cs_g[j] * bb;
                }
                const double a = H[(size_t)k * restart + k], bb = H[(size_t)(k + 1) * restart + k];
                const double rr = std::hypot(a, bb);
                cs_g[k] = rr > 0 ? a / rr : 1.0;
                sn_g[k] = rr > 0 ? bb / rr : 0.0;
                H[(size_t)k * restart + k] = rr;
                H[(size_t)(k + 1) * restart + k] = 0.0;
                gvec[k + 1] = -sn_g[k] * gvec[k];
                gvec[k] = cs_g[k] * gvec[k];
                ++inner_total;
                // Inner tolerance: each GMRES solve only has to shrink the
                // correction's residual by 1e-4; the FP64 outer loop does the rest.
                if (std::fabs(gvec[k + 1]) <= 1e-4 * beta || hn == 0.0) {
                    ++k;
                    break;
                }
            }
            // y = H^-1 g (upper triangular k x k), d = V y, x += d.
            for (int i = k - 1; i >= 0; --i) {
                double s = gvec[i];
                for (int j = i + 1; j < k; ++j) s -= H[(size_t)i * restart + j] * y[j];
                y[i] = s / H[(size_t)i * restart + i];
            }
            for (int j = 0; j < k; ++j)
                NMX_CUBLAS_TRY(cublasDaxpy(R.h, n, &y[j], Vk + (size_t)j * n, 1, x, 1));
        }
        // r = b - A x; norms.
        NMX_CUDA_TRY(cudaMemsetAsync(R.norms + 1, 0, 2 * sizeof(unsigned long long), st));
        residual_kernel<<<wb, threads, 0, st>>>(A, lda, n, x, b, R.r, R.norms + 1);
        absmax_kernel<<<std::min(vb, 1024), threads, 0, st>>>(x, n, R.norms + 2);
        NMX_CUDA_TRY(cudaGetLastError());
        NMX_CUDA_TRY(cudaMemcpyAsync(hnorm, R.norms, sizeof hnorm, cudaMemcpyDeviceToHost, st));
        NMX_CUDA_TRY(cudaStreamSynchronize(st));
        const double rn = bits_to_double(hnorm[1]), xn = bits_to_double(hnorm[2]),
                     bn = bits_to_double(hnorm[3]);
        berr = rn / (normA * xn + bn);
        int terr[6] = {0, 0, 0, 0, 0, 0};
        NMX_CUDA_TRY(cudaMemcpy(terr, R.counters, sizeof terr, cudaMemcpyDeviceToHost));
        if (terr[2] || terr[5]) {
            set_error("triangular solve: a bounded wait expired");
            return NMX_ERR_INTERNAL;
        }
        if (berr <= tol || !std::isfinite(berr)) break;
        // Plain refinement that stops contracting hands over to GMRES-IR when allowed.
        if (!use_gmres && (mode & NMX_IR_AUTO) && berr > 0.5 * prev) use_gmres = true;
        // Give up after 8 steps in a row without halving the backward error.
        if (berr > 0.5 * best_berr) {
            if (++stalled >= 8) break;
        } else {
            stalled = 0;
            best_berr = berr;
        }
        prev = berr;
    }
    NMX_CUDA_TRY(cudaEventRecord(e2, st));
    NMX_CUDA_TRY(cudaEventSynchronize(e2));
    if (stats) {
        float f_ms = 0, r_ms = 0;
        cudaEventElapsedTime(&f_ms, e0, e1);
        cudaEventElapsedTime(&r_ms, e1, e2);
        stats->iterations = std::min(it, max_iter);
        stats->gmres_iterations = inner_total;
        stats->converged = berr <= tol ? 1 : 0;
        stats->info = hinfo;
        stats->backward_error = berr;
        stats->factor_ms = f_ms;
        stats->refine_ms = r_ms;
        stats->used_gmres = use_gmres ? 1 : 0;
        stats->reserved = 0;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    return 0;
}

}  // namespace nmx

extern "C" NMX_API int nmx_gesv_ir_f64(nmx_ctx ctx, int64_t n, const double *A, int64_t lda,
                                       const double *b, double *x, int mode, double tol,
                                       int max_iter, nmx_ir_stats *stats, void *stream) {
    return nmx::gesv_ir(ctx, n, A, lda, b, x, mode, tol, max_iter, stats, stream);
}
