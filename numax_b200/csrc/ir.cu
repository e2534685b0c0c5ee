// Mixed-precision LU solve with iterative refinement (sm_100a).
//
// Not in numax (its GPU path is FP32-only and has no refinement); the
// north-star addition for the large solve.  A (FP64, row-major) is factored
// once in low precision and the solution is refined in FP64:
//
//   W = (float) R A C        R, C power-of-two row/column scalings (exact;
//                            FP16 factors only, which need the range)
//   P W = L U                the LU of dense_lu.cu (tournament pivoting,
//                            look-ahead) with its trailing updates on the
//                            tensor cores: BF16 or FP16 operands, or BF16
//                            hi/lo splits (BF16X3, ~16 bits) or hi/mid/lo
//                            splits (BF16X6, FP32's 24 bits), FP32 accumulate
//   x = 0, r = b
//   repeat: d = C U^-1 L^-1 P R r   (triangular solves read the factors,
//                                    arithmetic in FP64)
//           x += d; r = b - A x (FP64 GEMV over the original A)
//   until ||r||_inf / (||A||_inf ||x||_inf + ||b||_inf) <= tol
//
// GMRES-IR (Carson & Higham, SIAM J. Sci. Comput. 40(2), 2018) replaces the
// correction solve by GMRES on the left-preconditioned system
// (C U^-1 L^-1 P R A) d = C U^-1 L^-1 P R r, in FP64 with A applied in FP64.
// The whole Arnoldi step stays on the device: the matrix-vector product and
// the two triangular solves, classical Gram-Schmidt twice (CGS2) as per-CTA
// partial dot products reduced in a fixed order, the norm, the Givens
// rotation of the new Hessenberg column and the convergence test run as
// kernels that read and write a device-resident state; a step whose state
// says "done" returns at once, so the host launches steps in chunks and
// reads the state once per chunk.
//
// A refinement that cannot converge at its precision (the backward error
// stops halving, or GMRES stops reducing its residual) hands over, with
// NMX_IR_AUTO, from plain refinement to GMRES-IR, and with NMX_IR_ESCALATE
// refactors one level up (BF16 or FP16 -> BF16X3 -> BF16X6 -> FP64) and
// refines on from the best iterate so far.  The iterate with the smallest
// backward error is the one returned.
//
// The single-right-hand-side triangular solves are one persistent kernel
// each: CTAs take 64-row blocks in order from an atomic counter, stream the
// block's row segments left of the diagonal as the solution blocks they need
// become ready (a release/acquire counter of finished blocks), then solve the
// 64 x 64 diagonal block.  Every wait is bounded.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <type_traits>
#include <vector>

#include "dense_common.cuh"
#include "gemm_tc.cuh"

namespace nmx {

constexpr int kTrsvRB = 64;
constexpr int kTrsvThreads = 256;
constexpr int kTrsvPitch = kTrsvRB + 4;
constexpr long long kTrsvSpin = 1ll << 25;
template <typename TF>
constexpr size_t trsv_smem() {
    return (sizeof(double) + sizeof(TF)) * kTrsvRB * kTrsvPitch;
}

__device__ __forceinline__ int ld_acquire_i32(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_i32(int *p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Inverse of every 64 x 64 diagonal block of the lower (UPPER = false; unit
// diagonal when UNIT) or upper (UPPER = true) triangle of the factor F (FP32
// or FP64), in FP64:
// one CTA per block, thread j forms column j of the inverse by substitution.
// Computed once per factorization; it turns each block's serial substitution
// in the triangular solves into a 64 x 64 matrix-vector product.
template <typename TF, bool UPPER, bool UNIT = true>
__global__ void __launch_bounds__(kTrsvRB)
    diag_inverse_kernel(const TF *F, int64_t ldf, int n, double *Inv) {
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
                x[i] = (i < rows) ? (UNIT ? s : s / D[i][i]) : 0.0;
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

__device__ __forceinline__ void cp_async_n(unsigned dst, const void *src, int bytes) {
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_16(unsigned dst, const void *src) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all_() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <typename TF>
struct Pair;
template <>
struct Pair<float> {
    using type = float2;
};
template <>
struct Pair<double> {
    using type = double2;
};

// Solve with the unit-lower (UPPER = false) or upper (UPPER = true) triangle
// of the factor F (n x n, ldf; FP32 or FP64) in place on the FP64 vector x,
// using the precomputed FP64 inverses Inv of its 64 x 64 diagonal blocks.
// counter[0]: block ticket, counter[1]: blocks finished, counter[2]: error.
// `stop` (may be null): when it reads nonzero at entry the kernel does
// nothing (a finished GMRES step).  `out` (may be null): also writes
// out[i] = cs[i] x[i] as each block finishes.
//
// A CTA takes 64-row blocks in solve order.  It accumulates the block's row
// segments against the solution blocks finished so far as they appear, all
// but the adjacent one (the block finished just before it); meanwhile the
// F tile against that adjacent block and the block's Inv are copied into
// shared memory asynchronously.  So once the adjacent block is released,
// what remains on the chain from block to block is one 64-value read of x,
// two 64 x 64 products out of shared memory, and the release.
template <typename TF, bool UPPER>
__global__ void __launch_bounds__(kTrsvThreads)
    trsv_kernel(const TF *F, int64_t ldf, int n, const double *Inv, double *x, int *counter,
                const int *stop, const double *cs, double *out) {
    using P2 = typename Pair<TF>::type;
    // Dynamic shared memory: Is[64][68] (Inv of this block, FP64) then
    // Ft[64][68] (the F tile against the adjacent block).  Row pitch 68 with
    // thread (i, part) reading columns part + 4m keeps both conflict-free.
    extern __shared__ __align__(16) unsigned char trsv_smem_raw[];
    auto Is = reinterpret_cast<double(*)[kTrsvPitch]>(trsv_smem_raw);
    auto Ft = reinterpret_cast<TF(*)[kTrsvPitch]>(trsv_smem_raw +
                                                   sizeof(double) * kTrsvRB * kTrsvPitch);
    __shared__ double accS[kTrsvRB], xs[kTrsvRB], ys[kTrsvRB];
    __shared__ int s_blk, s_avail;
    if (stop && *stop) return;
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
            // Two columns per lane (pair loads: c0 is a multiple of 64, rows
            // start on 8-element boundaries, x 16-byte aligned), the 8 rows
            // and 2 iterations in flight: this stream must keep ahead of the
            // chain of blocks, so it needs memory-level parallelism.
            int c = c0 + 2 * lane;
#pragma unroll 2
            for (; c + 1 < c1; c += 64) {
                const double2 xv = __ldcg(reinterpret_cast<const double2 *>(x + c));
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int i = min(8 * warp + q, rows - 1);
                    const P2 f = *reinterpret_cast<const P2 *>(F + (int64_t)(r0 + i) * ldf + c);
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
                    cp_async_n(ft0 + (unsigned)(i * kTrsvPitch + c) * (unsigned)sizeof(TF),
                               F + (int64_t)(r0 + i) * ldf + a0 + c, (int)sizeof(TF));
                else
                    Ft[i][c] = TF(0);
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
            if (part == 0 && i < rows) {
                x[r0 + i] = s;
                if (out) out[r0 + i] = cs[r0 + i] * s;
            }
        }
        __threadfence();
        __syncthreads();
        if (tid == 0) st_release_i32(&counter[1], ticket + 1);
    }
}

// One row of A times v (FP64), a warp per row; the lanes' sum on lane 0.
__device__ __forceinline__ double row_dot(const double *row, const double *v, int n, int lane) {
    double s0 = 0.0, s1 = 0.0, s2 = 0.0, s3 = 0.0;
    int c = lane;
    for (; c + 96 < n; c += 128) {
        s0 += row[c] * v[c];
        s1 += row[c + 32] * v[c + 32];
        s2 += row[c + 64] * v[c + 64];
        s3 += row[c + 96] * v[c + 96];
    }
    for (; c < n; c += 32) s0 += row[c] * v[c];
    double s = (s0 + s1) + (s2 + s3);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    return s;
}

// r = b - A x (FP64), one warp per row; rmax <- max |r_i| (as ordered bits).
__global__ void residual_kernel(const double *A, int64_t lda, int n, const double *x,
                                const double *b, double *r, unsigned long long *rmax) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double s = row_dot(A + (int64_t)warp * lda, x, n, lane);
    if (lane == 0) {
        const double v = b[warp] - s;
        r[warp] = v;
        atomicMax(rmax, (unsigned long long)__double_as_longlong(fabs(v)));
    }
}

// max_i sum_j |A_ij| (||A||_inf) and per-row max |A_ij|.
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
        rowmax[warp] = m;
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

// W = (TW)(R A C), W row-major with ldw.
template <typename TW>
__global__ void scale_copy_kernel(const double *A, int64_t lda, int n, const double *rs,
                                  const double *cs, TW *W, int64_t ldw) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * n) return;
    const int i = (int)(e / n), j = (int)(e - (int64_t)i * n);
    W[(int64_t)i * ldw + j] = (TW)(A[(int64_t)i * lda + j] * rs[i] * cs[j]);
}

// Symmetric scaling D = diag(2^-round(log2 sqrt(a_ii))) (1 for a
// non-positive or non-finite a_ii): D A D has its diagonal in [0.5, 2).
__global__ void sym_scale_kernel(const double *A, int64_t lda, int n, double *d) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        const double a = A[(int64_t)i * lda + i];
        d[i] = (a > 0.0 && isfinite(a)) ? exp2(-rint(0.5 * log2(a))) : 1.0;
    }
}

// Copy the lower triangle of the n x n factor W into its strict upper
// triangle transposed (upper = L^T), 32 x 32 tiles through shared memory so
// that both the reads and the writes run along rows.  Tile (I, J), J <= I,
// is read and written to (J, I); a diagonal tile keeps its lower half.
template <typename T>
__global__ void __launch_bounds__(256) mirror_lower_kernel(T *W, int64_t ldw, int n) {
    __shared__ T t[32][33];
    const int I = blockIdx.y, J = blockIdx.x;
    if (J > I) return;
    const int tx = threadIdx.x & 31, ty = threadIdx.x >> 5;
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = 32 * I + ty + 8 * k, c = 32 * J + tx;
        t[ty + 8 * k][tx] = (r < n && c < n && c <= r) ? W[(int64_t)r * ldw + c] : T(0);
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int r = 32 * J + ty + 8 * k, c = 32 * I + tx;  // destination (r, c) = source (c, r)
        if (r < n && c < n && c > r) W[(int64_t)r * ldw + c] = t[tx][ty + 8 * k];
    }
}

__global__ void iota_kernel(int *p, int n) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) {
        p[i] = i;
        p[n + i] = i;
    }
}

// v[i] = s[perm[i]] * rs[perm[i]]  (apply P R to a vector).
__global__ void permute_scale_kernel(const double *s, const int *perm, const double *rs, int n,
                                     double *v) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) v[i] = s[perm[i]] * rs[perm[i]];
}

__global__ void add_kernel(const double *v, int n, double *x) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) x[i] += v[i];
}

// ---- GMRES on the device ------------------------------------------------

constexpr int kRestart = 200;    // Krylov basis size per GMRES cycle
constexpr int kGmresChunk = 6;   // Arnoldi steps launched between host reads
constexpr int kSlowStep = 32;    // step at which a slow cycle is abandoned
constexpr int kCgsThreads = 256;

// flag: 0 running, 1 converged, 2 breakdown (the Krylov space is invariant:
// the least-squares solution is exact), 3 basis full, 4 too slow (after
// kSlowStep steps the residual has not dropped tenfold).
struct GmresState {
    int flag;
    int k;        // Arnoldi steps completed (basis vectors V_0 .. V_k)
    int ky;       // length of y after the solve
    int slow_at;  // step of the "too slow" test (0: none)
    double beta, tol, inv_hn, pad2;
    double H[(kRestart + 1) * kRestart];  // H[j * kRestart + k]
    double cs[kRestart], sn[kRestart], g[kRestart + 1], y[kRestart], hcur[kRestart + 1];
};

// out[pinv[i]] = rs[i] (A V_k)[i]: P R A v with v the newest basis vector.
__global__ void gmres_matvec_kernel(const double *A, int64_t lda, int n, const double *V,
                                    const GmresState *st, const double *rs, const int *pinv,
                                    double *out) {
    if (st->flag) return;
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    if (warp >= n) return;
    const double *v = V + (size_t)st->k * n;
    const double s = row_dot(A + (int64_t)warp * lda, v, n, lane);
    if (lane == 0) out[pinv[warp]] = rs[warp] * s;
}

// Stage rows [r0, r1) of w in shared memory.  part[g][j] = V_j[chunk] . w[chunk]
// for j <= k, a warp per j.
__device__ __forceinline__ void chunk_dots(const double *V, int n, const double *wsm, int r0,
                                           int len, int kc, double *part_row) {
    const int lane = threadIdx.x & 31, wp = threadIdx.x >> 5, nw = blockDim.x >> 5;
    for (int j = wp; j < kc; j += nw) {
        const double *vj = V + (size_t)j * n + r0;
        double s = 0.0;
        for (int i = lane; i < len; i += 32) s += vj[i] * wsm[i];
        for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (lane == 0) part_row[j] = s;
    }
}

__global__ void __launch_bounds__(kCgsThreads)
    cgs_dots_kernel(const double *V, int n, const double *w, int rows_per, const GmresState *st,
                    double *part) {
    if (st->flag) return;
    extern __shared__ double wsm[];
    const int g = blockIdx.x, r0 = g * rows_per, len = min(n, r0 + rows_per) - r0;
    for (int i = threadIdx.x; i < len; i += blockDim.x) wsm[i] = w[r0 + i];
    __syncthreads();
    chunk_dots(V, n, wsm, r0, len, st->k + 1, part + (size_t)g * (kRestart + 1));
}

// h_j = sum_g part[g][j] in chunk order; pass 0: H[:, k] = h, pass 1: H[:, k] += h.
__global__ void cgs_reduce_kernel(const double *part, int G, GmresState *st, int pass) {
    if (st->flag) return;
    const int k = st->k, j = threadIdx.x;
    if (j > k) return;
    double s = 0.0;
    for (int g = 0; g < G; ++g) s += part[(size_t)g * (kRestart + 1) + j];
    st->hcur[j] = s;
    st->H[j * kRestart + k] = pass ? st->H[j * kRestart + k] + s : s;
}

// w -= V h over the chunk.  mode 0: part[g][j] = V_j . w (the second pass's
// projections); mode 1: the new vector goes to V_{k+1} and part[g][0] =
// ||w||^2 over the chunk.
__global__ void __launch_bounds__(kCgsThreads)
    cgs_update_kernel(double *V, int n, double *w, int rows_per, const GmresState *st,
                      double *part, int mode) {
    if (st->flag) return;
    extern __shared__ double wsm[];
    __shared__ double h[kRestart + 1];
    __shared__ double red[kCgsThreads / 32];
    const int kc = st->k + 1;
    const int g = blockIdx.x, r0 = g * rows_per, len = min(n, r0 + rows_per) - r0;
    for (int j = threadIdx.x; j < kc; j += blockDim.x) h[j] = st->hcur[j];
    __syncthreads();
    double *dst = mode ? V + (size_t)kc * n : w;
    double ss = 0.0;
    for (int i = threadIdx.x; i < len; i += blockDim.x) {
        double s = w[r0 + i];
        for (int j = 0; j < kc; ++j) s -= V[(size_t)j * n + r0 + i] * h[j];
        wsm[i] = s;
        dst[r0 + i] = s;
        ss += s * s;
    }
    if (mode == 0) {
        __syncthreads();
        chunk_dots(V, n, wsm, r0, len, kc, part + (size_t)g * (kRestart + 1));
    } else {
        for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
        if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ss;
        __syncthreads();
        if (threadIdx.x == 0) {
            double t = 0.0;
            for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
            part[(size_t)g * (kRestart + 1)] = t;
        }
    }
}

// part[g][0] = ||v||^2 over chunk g (the first basis vector's norm).
__global__ void __launch_bounds__(kCgsThreads)
    chunk_norm2_kernel(const double *v, int n, int rows_per, double *part) {
    __shared__ double red[kCgsThreads / 32];
    const int g = blockIdx.x, r0 = g * rows_per, r1 = min(n, r0 + rows_per);
    double ss = 0.0;
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) ss += v[i] * v[i];
    for (int o = 16; o > 0; o >>= 1) ss += __shfl_xor_sync(0xffffffffu, ss, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ss;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int q = 0; q < (int)(blockDim.x >> 5); ++q) t += red[q];
        part[(size_t)g * (kRestart + 1)] = t;
    }
}

// One thread: beta = ||z0||, g = beta e1, k = 0.
__global__ void gmres_start_kernel(const double *part, int G, GmresState *st, double tol,
                                   int slow_at) {
    double ss = 0.0;
    for (int g = 0; g < G; ++g) ss += part[(size_t)g * (kRestart + 1)];
    const double beta = sqrt(ss);
    st->beta = beta;
    st->tol = tol;
    st->k = 0;
    st->ky = 0;
    st->slow_at = slow_at;
    st->g[0] = beta;
    st->inv_hn = beta > 0.0 ? 1.0 / beta : 0.0;
    st->flag = (beta > 0.0 && isfinite(beta)) ? 0 : 2;
}

// One thread: h_{k+1,k} = ||w||, the earlier rotations applied to column k of
// H, a new rotation zeroing h_{k+1,k}, g updated, the stopping tests.
__global__ void arnoldi_finish_kernel(const double *part, int G, GmresState *st) {
    if (st->flag) return;
    const int k = st->k;
    double ss = 0.0;
    for (int g = 0; g < G; ++g) ss += part[(size_t)g * (kRestart + 1)];
    const double hn = sqrt(ss);
    double *H = st->H;
    for (int j = 0; j < k; ++j) {
        const double a = H[j * kRestart + k], b = H[(j + 1) * kRestart + k];
        H[j * kRestart + k] = st->cs[j] * a + st->sn[j] * b;
        H[(j + 1) * kRestart + k] = -st->sn[j] * a + st->cs[j] * b;
    }
    const double a = H[k * kRestart + k];
    const double rr = hypot(a, hn);
    const double c = rr > 0.0 ? a / rr : 1.0, s = rr > 0.0 ? hn / rr : 0.0;
    st->cs[k] = c;
    st->sn[k] = s;
    H[k * kRestart + k] = rr;
    st->g[k + 1] = -s * st->g[k];
    st->g[k] = c * st->g[k];
    st->k = k + 1;
    st->inv_hn = hn > 0.0 ? 1.0 / hn : 0.0;
    const double res = fabs(st->g[k + 1]);
    if (res <= st->tol * st->beta)
        st->flag = 1;
    else if (!(hn > 0.0) || !isfinite(hn))
        st->flag = 2;
    else if (k + 1 == kRestart)
        st->flag = 3;
    else if (k + 1 == st->slow_at && res > 0.1 * st->beta)
        st->flag = 4;
}

// V_k *= inv_hn (k already counts the new vector).
__global__ void scale_basis_kernel(double *V, int n, const GmresState *st) {
    if (st->flag) return;
    double *v = V + (size_t)st->k * n;
    const double s = st->inv_hn;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) v[i] *= s;
}

// One thread: y = R^-1 g over the leading k x k triangle of the rotated H,
// shortened at the first diagonal that is negligible against the largest
// (a least-squares solution of the leading block instead of a blow-up).
__global__ void gmres_solve_kernel(GmresState *st) {
    const int k = st->k;
    const double *H = st->H;
    double hmax = 0.0;
    for (int i = 0; i < k; ++i) hmax = fmax(hmax, fabs(H[i * kRestart + i]));
    int kk = k;
    for (int i = 0; i < k; ++i)
        if (!(fabs(H[i * kRestart + i]) > 1e-14 * hmax)) {
            kk = i;
            break;
        }
    for (int i = kk - 1; i >= 0; --i) {
        double s = st->g[i];
        for (int j = i + 1; j < kk; ++j) s -= H[i * kRestart + j] * st->y[j];
        st->y[i] = s / H[i * kRestart + i];
    }
    st->ky = kk;
}

// x += V y.
__global__ void gmres_update_kernel(const double *V, int n, const GmresState *st, double *x) {
    const int ky = st->ky;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        double s = 0.0;
        for (int j = 0; j < ky; ++j) s += V[(size_t)j * n + i] * st->y[j];
        x[i] += s;
    }
}

// ---- host side ----------------------------------------------------------

// Precision levels, in escalation order.
enum IrLevel { kLvBF16 = 0, kLvFP16, kLvBF16X3, kLvBF16X6, kLvFP32, kLvFP64 };

static int level_of(int prec) {
    switch (prec) {
        case NMX_IR_BF16: return kLvBF16;
        case NMX_IR_FP16: return kLvFP16;
        case NMX_IR_BF16X3: return kLvBF16X3;
        case NMX_IR_BF16X6: return kLvBF16X6;
        case NMX_IR_FP32: return kLvFP32;
        default: return kLvFP64;
    }
}
static int prec_of(int level) {
    static const int p[] = {NMX_IR_BF16, NMX_IR_FP16, NMX_IR_BF16X3, NMX_IR_BF16X6, NMX_IR_FP32,
                            NMX_IR_FP64};
    return p[level];
}
// The next, more accurate level: 8-bit and 11-bit factors go to ~16 bits,
// then to FP32's 24 bits, then to FP64 itself.
static int next_level(int level) {
    switch (level) {
        case kLvBF16:
        case kLvFP16: return kLvBF16X3;
        case kLvBF16X3: return kLvBF16X6;
        default: return kLvFP64;
    }
}
static int gemm_precision(int level) {
    switch (level) {
        case kLvBF16: return NMX_PREC_BF16;
        case kLvFP16: return NMX_PREC_FP16;
        case kLvBF16X3: return NMX_PREC_BF16X3;
        case kLvBF16X6: return NMX_PREC_BF16X6;
        default: return 0;
    }
}

struct IrRun {
    nmx_ctx ctx;
    cudaStream_t st;
    bool spd = false;  // Cholesky factors (A symmetric positive definite)
    int n;
    const double *A;
    int64_t lda;
    int level = -1;
    float *W = nullptr;     // FP32 factors (levels below FP64)
    double *W64 = nullptr;  // FP64 factors
    int64_t ldw;
    int *perm, *pinv;
    double *rs, *cs, *v, *r, *tmp, *w, *rowmax, *xbest;
    int *counters;  // 3 per triangular solve
    double *invL, *invU;  // inverses of the 64 x 64 diagonal blocks of L and U
    unsigned long long *norms;  // [0] ||A||_inf, [1] ||r||, [2] ||x||, [3] ||b||
    int32_t *ipiv, *info_d;
    double *V = nullptr;   // Krylov basis, kRestart + 1 vectors of n
    double *part = nullptr;
    GmresState *gst = nullptr;
    int G = 1, rows_per = 1;  // chunks of the Gram-Schmidt kernels
};

static double bits_to_double(unsigned long long u) {
    double d;
    std::memcpy(&d, &u, sizeof d);
    return d;
}

static size_t ir_vec_bytes(int64_t n) {
    return sizeof(double) * (size_t)n * 9 + sizeof(int) * (size_t)n * 4 + 4096;
}
static size_t ir_krylov_bytes(int64_t n, int G) {
    return sizeof(double) * ((size_t)n * (kRestart + 1) + (size_t)G * (kRestart + 1)) +
           sizeof(GmresState) + 1024;
}

// The largest tensor-core update of the FP32 factorization: look-ahead
// panels of nb columns (tournament leaves, order >= 2 nb; the same decision
// getrf_run makes) bound its inner dimension at nb; otherwise the recursion's
// largest update is about half the order.
static size_t ir_gemm_ws_bytes(nmx_ctx ctx, int64_t n, int prec, bool spd = false) {
    if (!prec) return 0;
    if (spd) {  // the Cholesky recursion: the largest update is the first SYRK
        const int64_t half = (n / 2 + 31) / 32 * 32;
        return tc_gemm_workspace_bytes(n - half, n - half, std::max<int64_t>(half, 1), prec) + 4096;
    }
    const bool tournament = ctx->tune_lu_tournament != 0 && n <= tournament_max_rows();
    const int64_t want = ctx->tune_lu_lookahead >= 0 ? ctx->tune_lu_lookahead : 256;
    const int64_t nb = std::min<int64_t>(1024, want / 32 * 32);
    if (tournament && nb >= 64 && n >= 2 * nb)
        return tc_gemm_workspace_bytes(n, n, nb, prec) + 4096;
    const int64_t half = (n / 2 + 31) / 32 * 32;
    return tc_gemm_workspace_bytes(n - half, n - half, std::max<int64_t>(half, 1), prec) + 4096;
}

// Every buffer a solve at `level` (and, when escalating, at the levels above
// it) needs, grown now.
static int ir_reserve(nmx_ctx ctx, int64_t n, int level, bool escalate, bool spd) {
    void *p = nullptr;
    const int64_t ldw = (n + 7) / 8 * 8;
    const int G = std::max(1, std::min<int>(2 * ctx->sm_count, (int)ceil_div(n, 256)));
    NMX_TRY(ctx->ensure_slot(kWsVec, ir_vec_bytes(n), &p));
    NMX_TRY(ctx->ensure_slot(kWsKrylov, ir_krylov_bytes(n, G), &p));
    NMX_TRY(ctx->ensure_slot(kWsBest, sizeof(double) * (size_t)n + 256, &p));
    const int NB = (int)ceil_div(n, kTrsvRB);
    NMX_TRY(ctx->ensure_slot(kWsInv, sizeof(double) * (size_t)NB * kTrsvRB * kTrsvRB * 2 + 256, &p));
    size_t gemm_ws = 0;
    bool need32 = false, need64 = false;
    for (int lv = level;; lv = next_level(lv)) {
        if (lv == kLvFP64)
            need64 = true;
        else
            need32 = true;
        gemm_ws = std::max(gemm_ws, ir_gemm_ws_bytes(ctx, n, gemm_precision(lv), spd));
        if (!escalate || lv == kLvFP64) break;
    }
    if (need32) NMX_TRY(ctx->ensure_slot(kWsWork, sizeof(float) * (size_t)n * ldw + 256, &p));
    if (need64) NMX_TRY(ctx->ensure_slot(kWsWork64, sizeof(double) * (size_t)n * ldw + 256, &p));
    if (gemm_ws) NMX_TRY(ctx->ensure_slot(kWsGemm16, gemm_ws, &p));
    return 0;
}

// v := U^-1 L^-1 v with the current level's factors, arithmetic in FP64;
// with `out`, also out = C v.  `stop`: the GMRES state's flag, or null.
static int lu_solve_inplace(IrRun &R, double *v, const int *stop, double *out) {
    const int NB = (R.n + kTrsvRB - 1) / kTrsvRB;
    const int want = R.ctx->tune_ir_trsv_ctas > 0 ? (int)R.ctx->tune_ir_trsv_ctas
                                                  : 2 * R.ctx->sm_count;
    const int grid = std::max(1, std::min(NB, want));
    static bool attr_set[64][2] = {};
    const int f64 = R.level == kLvFP64 ? 1 : 0;
    if (R.ctx->device < 64 && !attr_set[R.ctx->device][f64]) {
        if (f64) {
            NMX_CUDA_TRY(cudaFuncSetAttribute(trsv_kernel<double, false>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)trsv_smem<double>()));
            NMX_CUDA_TRY(cudaFuncSetAttribute(trsv_kernel<double, true>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)trsv_smem<double>()));
        } else {
            NMX_CUDA_TRY(cudaFuncSetAttribute(trsv_kernel<float, false>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)trsv_smem<float>()));
            NMX_CUDA_TRY(cudaFuncSetAttribute(trsv_kernel<float, true>,
                                              cudaFuncAttributeMaxDynamicSharedMemorySize,
                                              (int)trsv_smem<float>()));
        }
        attr_set[R.ctx->device][f64] = true;
    }
    NMX_CUDA_TRY(cudaMemsetAsync(R.counters, 0, 6 * sizeof(int), R.st));
    if (f64) {
        trsv_kernel<double, false><<<grid, kTrsvThreads, trsv_smem<double>(), R.st>>>(
            R.W64, R.ldw, R.n, R.invL, v, R.counters, stop, nullptr, nullptr);
        trsv_kernel<double, true><<<grid, kTrsvThreads, trsv_smem<double>(), R.st>>>(
            R.W64, R.ldw, R.n, R.invU, v, R.counters + 3, stop, R.cs, out);
    } else {
        trsv_kernel<float, false><<<grid, kTrsvThreads, trsv_smem<float>(), R.st>>>(
            R.W, R.ldw, R.n, R.invL, v, R.counters, stop, nullptr, nullptr);
        trsv_kernel<float, true><<<grid, kTrsvThreads, trsv_smem<float>(), R.st>>>(
            R.W, R.ldw, R.n, R.invU, v, R.counters + 3, stop, R.cs, out);
    }
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

// out = C U^-1 L^-1 P R in   (the preconditioned correction of one residual).
static int precond_apply(IrRun &R, const double *in, double *out) {
    const int threads = 256, blocks = (int)ceil_div(R.n, threads);
    permute_scale_kernel<<<blocks, threads, 0, R.st>>>(in, R.perm, R.rs, R.n, R.tmp);
    NMX_CUDA_TRY(cudaGetLastError());
    return lu_solve_inplace(R, R.tmp, nullptr, out);
}

// Factor A at `level` into R's buffers: scalings, the copy, the LU, the
// diagonal-block inverses (then `done` is recorded, when given), and the
// permutation (read back to the host).
static int ir_factor(IrRun &R, int level, int32_t *hinfo, cudaEvent_t done) {
    nmx_ctx ctx = R.ctx;
    cudaStream_t st = R.st;
    const int n = R.n;
    const int threads = 256;
    const int vb = (int)ceil_div(n, threads);
    const int wb = (int)ceil_div((int64_t)n * 32, threads);
    void *p = nullptr;
    R.level = level;
    // ||A||_inf and the row maxima (also the row scales' input).
    NMX_CUDA_TRY(cudaMemsetAsync(R.norms, 0, sizeof(unsigned long long), st));
    row_norms_kernel<<<wb, threads, 0, st>>>(R.A, R.lda, n, R.norms, R.rowmax);
    const int equil = level == kLvFP16 ? 1 : 0;
    if (R.spd) {
        // Symmetric scaling D A D (every level: it keeps the Cholesky's
        // pivots near 1), no permutation.
        sym_scale_kernel<<<vb, threads, 0, st>>>(R.A, R.lda, n, R.rs);
        NMX_CUDA_TRY(cudaMemcpyAsync(R.cs, R.rs, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    } else {
        row_scale_kernel<<<vb, threads, 0, st>>>(R.rowmax, n, R.rs, equil);
    }
    if (R.spd) {
    } else if (equil) {
        // The column maxima go through R.tmp's bits (free until the solve).
        unsigned long long *cmax = reinterpret_cast<unsigned long long *>(R.tmp);
        NMX_CUDA_TRY(cudaMemsetAsync(cmax, 0, sizeof(double) * n, st));
        col_max_kernel<<<dim3(vb, kColChunks), threads, 0, st>>>(R.A, R.lda, n, R.rs, cmax);
        col_scale_kernel<<<vb, threads, 0, st>>>(cmax, n, R.cs, 1);
    } else {
        col_scale_kernel<<<vb, threads, 0, st>>>(nullptr, n, R.cs, 0);
    }
    NMX_CUDA_TRY(cudaGetLastError());
    const unsigned cb = (unsigned)ceil_div((int64_t)n * n, threads);
    if (level == kLvFP64) {
        NMX_TRY(ctx->ensure_slot(kWsWork64, sizeof(double) * (size_t)n * R.ldw + 256, &p));
        R.W64 = static_cast<double *>(p);
        scale_copy_kernel<double><<<cb, threads, 0, st>>>(R.A, R.lda, n, R.rs, R.cs, R.W64, R.ldw);
        NMX_CUDA_TRY(cudaGetLastError());
        GemmSub gs;
        gs.st = st;
        if (R.spd)
            NMX_TRY(potrf_run<double>(gs, n, R.W64, R.ldw, R.info_d));
        else
            NMX_TRY(getrf_run<double>(ctx, gs, n, R.W64, R.ldw, R.ipiv, R.info_d, false));
    } else {
        NMX_TRY(ctx->ensure_slot(kWsWork, sizeof(float) * (size_t)n * R.ldw + 256, &p));
        R.W = static_cast<float *>(p);
        scale_copy_kernel<float><<<cb, threads, 0, st>>>(R.A, R.lda, n, R.rs, R.cs, R.W, R.ldw);
        NMX_CUDA_TRY(cudaGetLastError());
        GemmSub gs;
        gs.st = st;
        gs.precision = gemm_precision(level);
        if (ctx->tune_ir_tc_min >= 0) gs.tc_min = ctx->tune_ir_tc_min;
        if (gs.precision) {
            gs.ws_bytes = ir_gemm_ws_bytes(ctx, n, gs.precision, R.spd);
            NMX_TRY(ctx->ensure_slot(kWsGemm16, gs.ws_bytes, &gs.ws));
        }
        if (R.spd)
            NMX_TRY(potrf_run<float>(gs, n, R.W, R.ldw, R.info_d));
        else
            NMX_TRY(getrf_run<float>(ctx, gs, n, R.W, R.ldw, R.ipiv, R.info_d,
                                     ctx->tune_lu_tournament != 0));
    }
    if (R.spd) {  // upper = L^T, so that the two solves read rows
        const dim3 mg((unsigned)ceil_div(n, 32), (unsigned)ceil_div(n, 32));
        if (level == kLvFP64)
            mirror_lower_kernel<double><<<mg, 256, 0, st>>>(R.W64, R.ldw, n);
        else
            mirror_lower_kernel<float><<<mg, 256, 0, st>>>(R.W, R.ldw, n);
        NMX_CUDA_TRY(cudaGetLastError());
    }
    // Inverses of the diagonal blocks of L and U for the triangular solves.
    const int NB = (n + kTrsvRB - 1) / kTrsvRB;
    NMX_TRY(ctx->ensure_slot(kWsInv, sizeof(double) * (size_t)NB * kTrsvRB * kTrsvRB * 2 + 256, &p));
    R.invL = static_cast<double *>(p);
    R.invU = R.invL + (size_t)NB * kTrsvRB * kTrsvRB;
    if (level == kLvFP64) {
        if (R.spd)
            diag_inverse_kernel<double, false, false><<<NB, kTrsvRB, 0, st>>>(R.W64, R.ldw, n, R.invL);
        else
            diag_inverse_kernel<double, false><<<NB, kTrsvRB, 0, st>>>(R.W64, R.ldw, n, R.invL);
        diag_inverse_kernel<double, true><<<NB, kTrsvRB, 0, st>>>(R.W64, R.ldw, n, R.invU);
    } else {
        if (R.spd)
            diag_inverse_kernel<float, false, false><<<NB, kTrsvRB, 0, st>>>(R.W, R.ldw, n, R.invL);
        else
            diag_inverse_kernel<float, false><<<NB, kTrsvRB, 0, st>>>(R.W, R.ldw, n, R.invL);
        diag_inverse_kernel<float, true><<<NB, kTrsvRB, 0, st>>>(R.W, R.ldw, n, R.invU);
    }
    NMX_CUDA_TRY(cudaGetLastError());
    if (done) NMX_CUDA_TRY(cudaEventRecord(done, st));
    if (R.spd) {  // no pivoting: identity permutation
        *hinfo = 0;
        iota_kernel<<<(unsigned)ceil_div(n, threads), threads, 0, st>>>(R.perm, n);
        NMX_CUDA_TRY(cudaGetLastError());
        NMX_CUDA_TRY(cudaMemcpyAsync(hinfo, R.info_d, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        NMX_CUDA_TRY(cudaStreamSynchronize(st));
        return 0;
    }
    // Pivots -> permutation and its inverse on the host (the interchanges
    // compose in order).
    std::vector<int32_t> hp(n), perm(2 * (size_t)n);
    NMX_CUDA_TRY(cudaMemcpyAsync(hp.data(), R.ipiv, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, st));
    NMX_CUDA_TRY(cudaMemcpyAsync(hinfo, R.info_d, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    NMX_CUDA_TRY(cudaStreamSynchronize(st));
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int j = 0; j < n; ++j)
        if (hp[j] != j) std::swap(perm[j], perm[hp[j]]);
    for (int i = 0; i < n; ++i) perm[n + perm[i]] = i;
    NMX_CUDA_TRY(cudaMemcpyAsync(R.perm, perm.data(), sizeof(int32_t) * 2 * (size_t)n,
                                 cudaMemcpyHostToDevice, st));
    // The copy reads pageable host memory: it is staged before the call
    // returns, so `perm` may go out of scope.
    return 0;
}

// One GMRES cycle on M^-1 A d = M^-1 r from d = 0, then x += d.  *steps gets
// the Arnoldi steps taken, *flag the state's final flag.  `give_up_early`:
// end a cycle that has not cut its residual tenfold by step kSlowStep (when
// a more accurate factorization can take over).
static int gmres_cycle(IrRun &R, double *x, bool give_up_early, int *steps, int *flag) {
    cudaStream_t st = R.st;
    const int n = R.n;
    const int threads = 256;
    const int wb = (int)ceil_div((int64_t)n * 32, threads);
    const size_t wsm = sizeof(double) * (size_t)R.rows_per;
    // z0 = M^-1 r -> V_0, beta, V_0 /= beta.
    NMX_TRY(precond_apply(R, R.r, R.V));
    chunk_norm2_kernel<<<R.G, kCgsThreads, 0, st>>>(R.V, n, R.rows_per, R.part);
    gmres_start_kernel<<<1, 1, 0, st>>>(R.part, R.G, R.gst, 1e-4, give_up_early ? kSlowStep : 0);
    scale_basis_kernel<<<(unsigned)std::min<int64_t>(ceil_div(n, threads), 1024), threads, 0, st>>>(
        R.V, n, R.gst);
    NMX_CUDA_TRY(cudaGetLastError());
    int hstate[2] = {0, 0};
    for (int s = 0; s < kRestart;) {
        const int chunk = std::min(kGmresChunk, kRestart - s);
        for (int c = 0; c < chunk; ++c) {
            gmres_matvec_kernel<<<wb, threads, 0, st>>>(R.A, R.lda, n, R.V, R.gst, R.rs, R.pinv,
                                                        R.tmp);
            NMX_TRY(lu_solve_inplace(R, R.tmp, &R.gst->flag, R.w));
            cgs_dots_kernel<<<R.G, kCgsThreads, wsm, st>>>(R.V, n, R.w, R.rows_per, R.gst, R.part);
            cgs_reduce_kernel<<<1, kRestart + 1, 0, st>>>(R.part, R.G, R.gst, 0);
            cgs_update_kernel<<<R.G, kCgsThreads, wsm, st>>>(R.V, n, R.w, R.rows_per, R.gst, R.part,
                                                             0);
            cgs_reduce_kernel<<<1, kRestart + 1, 0, st>>>(R.part, R.G, R.gst, 1);
            cgs_update_kernel<<<R.G, kCgsThreads, wsm, st>>>(R.V, n, R.w, R.rows_per, R.gst, R.part,
                                                             1);
            arnoldi_finish_kernel<<<1, 1, 0, st>>>(R.part, R.G, R.gst);
            scale_basis_kernel<<<(unsigned)std::min<int64_t>(ceil_div(n, threads), 1024), threads,
                                 0, st>>>(R.V, n, R.gst);
            NMX_CUDA_TRY(cudaGetLastError());
        }
        s += chunk;
        NMX_CUDA_TRY(cudaMemcpyAsync(hstate, R.gst, sizeof hstate, cudaMemcpyDeviceToHost, st));
        NMX_CUDA_TRY(cudaStreamSynchronize(st));
        if (hstate[0]) break;
    }
    gmres_solve_kernel<<<1, 1, 0, st>>>(R.gst);
    gmres_update_kernel<<<(unsigned)std::min<int64_t>(ceil_div(n, threads), 1024), threads, 0, st>>>(
        R.V, n, R.gst, x);
    NMX_CUDA_TRY(cudaGetLastError());
    *steps = hstate[1];
    *flag = hstate[0];
    return 0;
}

// r = b - A x and the backward error (synchronizes).
static int ir_residual(IrRun &R, const double *b, const double *x, double normA, double *berr) {
    cudaStream_t st = R.st;
    const int n = R.n, threads = 256;
    const int vb = (int)ceil_div(n, threads);
    const int wb = (int)ceil_div((int64_t)n * 32, threads);
    NMX_CUDA_TRY(cudaMemsetAsync(R.norms + 1, 0, 2 * sizeof(unsigned long long), st));
    residual_kernel<<<wb, threads, 0, st>>>(R.A, R.lda, n, x, b, R.r, R.norms + 1);
    absmax_kernel<<<std::min(vb, 1024), threads, 0, st>>>(x, n, R.norms + 2);
    NMX_CUDA_TRY(cudaGetLastError());
    unsigned long long hn[4];
    int terr[6] = {0, 0, 0, 0, 0, 0};
    NMX_CUDA_TRY(cudaMemcpyAsync(hn, R.norms, sizeof hn, cudaMemcpyDeviceToHost, st));
    NMX_CUDA_TRY(cudaMemcpyAsync(terr, R.counters, sizeof terr, cudaMemcpyDeviceToHost, st));
    NMX_CUDA_TRY(cudaStreamSynchronize(st));
    const double rn = bits_to_double(hn[1]), xn = bits_to_double(hn[2]), bn = bits_to_double(hn[3]);
    *berr = rn / (normA * xn + bn);
    if (terr[2] || terr[5]) {
        set_error("triangular solve: a bounded wait expired");
        return NMX_ERR_INTERNAL;
    }
    return 0;
}

static int gesv_ir(nmx_ctx ctx, int64_t n64, const double *A, int64_t lda, const double *b,
                   double *x, int mode, double tol, int max_iter, nmx_ir_stats *stats,
                   void *stream, bool spd) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(n64 >= 1 && n64 <= (1 << 17), 2, "n must be in 1..131072");
    NMX_ARG_CHECK(A != nullptr, 3, "A is NULL");
    NMX_ARG_CHECK(lda >= n64, 4, "lda < n");
    NMX_ARG_CHECK(b != nullptr, 5, "b is NULL");
    NMX_ARG_CHECK(x != nullptr, 6, "x is NULL");
    const int prec = mode & 0xF;
    NMX_ARG_CHECK(prec >= NMX_IR_BF16 && prec <= NMX_IR_FP64, 7,
                  "mode must be NMX_IR_BF16/FP16/FP32/BF16X3/BF16X6/FP64, optionally | "
                  "NMX_IR_GMRES / NMX_IR_AUTO / NMX_IR_ESCALATE");
    NMX_ARG_CHECK(tol >= 0.0, 8, "tol < 0");
    NMX_ARG_CHECK(max_iter >= 1 && max_iter <= 10000, 9, "max_iter must be in 1..10000");
    const bool force_gmres = (mode & NMX_IR_GMRES) != 0;
    const bool auto_gmres = (mode & NMX_IR_AUTO) != 0;
    const bool escalate = (mode & NMX_IR_ESCALATE) != 0;
    const int n = (int)n64;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    IrRun R;
    R.ctx = ctx;
    R.st = st;
    R.spd = spd;
    R.n = n;
    R.A = A;
    R.lda = lda;
    R.ldw = (n + 7) / 8 * 8;
    R.G = std::max(1, std::min<int>(2 * ctx->sm_count, (int)ceil_div(n, 256)));
    R.rows_per = (int)ceil_div(n, R.G);
    R.G = (int)ceil_div(n, R.rows_per);
    int level = level_of(prec);
    NMX_TRY(ir_reserve(ctx, n, level, escalate, spd));
    void *p = nullptr;
    NMX_TRY(ctx->ensure_slot(kWsVec, ir_vec_bytes(n), &p));
    char *vp = static_cast<char *>(p);
    R.norms = reinterpret_cast<unsigned long long *>(vp);
    R.counters = reinterpret_cast<int *>(vp + 256);
    R.info_d = R.counters + 16;
    double *dv = reinterpret_cast<double *>(vp + 1024);
    R.rs = dv;
    R.cs = dv + n;
    R.v = dv + 2 * (size_t)n;
    R.r = dv + 3 * (size_t)n;
    R.tmp = dv + 4 * (size_t)n;
    R.rowmax = dv + 5 * (size_t)n;
    R.w = dv + 6 * (size_t)n;
    R.perm = reinterpret_cast<int *>(dv + 9 * (size_t)n);
    R.pinv = R.perm + n;
    R.ipiv = R.pinv + n;
    NMX_TRY(ctx->ensure_slot(kWsKrylov, ir_krylov_bytes(n, R.G), &p));
    R.V = static_cast<double *>(p);
    R.part = R.V + (size_t)n * (kRestart + 1);
    R.gst = reinterpret_cast<GmresState *>(R.part + (size_t)R.G * (kRestart + 1));
    NMX_TRY(ctx->ensure_slot(kWsBest, sizeof(double) * (size_t)n + 256, &p));
    R.xbest = static_cast<double *>(p);
    const int threads = 256;
    const int vb = (int)ceil_div(n, threads);

    cudaEvent_t e0, e1, e2;
    NMX_CUDA_TRY(cudaEventCreate(&e0));
    NMX_CUDA_TRY(cudaEventCreate(&e1));
    NMX_CUDA_TRY(cudaEventCreate(&e2));
    struct EventsGuard {
        cudaEvent_t *e;
        ~EventsGuard() {
            for (int i = 0; i < 3; ++i) cudaEventDestroy(e[i]);
        }
    };
    cudaEvent_t evs[3] = {e0, e1, e2};
    EventsGuard eg{evs};
    NMX_CUDA_TRY(cudaEventRecord(e0, st));
    int32_t hinfo = 0;
    NMX_TRY(ir_factor(R, level, &hinfo, e1));
    unsigned long long hnorm0 = 0;
    NMX_CUDA_TRY(cudaMemcpyAsync(&hnorm0, R.norms, sizeof hnorm0, cudaMemcpyDeviceToHost, st));
    // ||b||_inf; x = 0, r = b.
    NMX_CUDA_TRY(cudaMemsetAsync(R.norms + 3, 0, sizeof(unsigned long long), st));
    absmax_kernel<<<std::min(vb, 1024), threads, 0, st>>>(b, n, R.norms + 3);
    NMX_CUDA_TRY(cudaMemsetAsync(x, 0, sizeof(double) * n, st));
    NMX_CUDA_TRY(cudaMemsetAsync(R.xbest, 0, sizeof(double) * n, st));
    NMX_CUDA_TRY(cudaMemcpyAsync(R.r, b, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    NMX_CUDA_TRY(cudaStreamSynchronize(st));
    const double normA = bits_to_double(hnorm0);

    double factor_extra_ms = 0.0;  // refactorizations after an escalation
    int it = 0, inner_total = 0, since_best = 0, level_steps = 0;
    double berr = INFINITY, prev = INFINITY, best = INFINITY;
    bool use_gmres = force_gmres, used_gmres = false;
    for (it = 1; it <= max_iter; ++it) {
        int gflag = 0;
        if (!use_gmres) {
            NMX_TRY(precond_apply(R, R.r, R.v));  // d = M^-1 r
            add_kernel<<<vb, threads, 0, st>>>(R.v, n, x);
            NMX_CUDA_TRY(cudaGetLastError());
        } else {
            int steps = 0;
            NMX_TRY(gmres_cycle(R, x, escalate && R.level != kLvFP64, &steps, &gflag));
            inner_total += steps;
            used_gmres = true;
        }
        ++level_steps;
        NMX_TRY(ir_residual(R, b, x, normA, &berr));
        if (berr < best) {
            if (best < INFINITY && berr > 0.5 * best)
                ++since_best;  // an improvement, but not a halving
            else
                since_best = 0;
            best = berr;
            NMX_CUDA_TRY(cudaMemcpyAsync(R.xbest, x, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
        } else {
            ++since_best;
        }
        if (best <= tol) break;
        // Does this precision still contract?  Plain refinement: the backward
        // error must halve per step; a GMRES cycle must reach its own
        // tolerance (or at least cut the backward error tenfold).
        bool stuck;
        if (!use_gmres)
            stuck = level_steps >= 2 && berr > 0.5 * prev;
        else
            stuck = (gflag == 4 || gflag == 3) ? berr > 0.1 * prev : berr > 0.5 * prev;
        stuck = stuck || !std::isfinite(berr);
        prev = berr;
        if (!stuck) continue;
        if (!use_gmres && (auto_gmres || force_gmres)) {
            use_gmres = true;  // hand over to GMRES-IR at the same precision
        } else if (escalate && R.level != kLvFP64) {
            // Refactor one level up and refine on from the best iterate.
            cudaEvent_t f0, f1;
            NMX_CUDA_TRY(cudaEventCreate(&f0));
            NMX_CUDA_TRY(cudaEventCreate(&f1));
            NMX_CUDA_TRY(cudaEventRecord(f0, st));
            int rc = ir_factor(R, next_level(R.level), &hinfo, f1);
            if (!rc) rc = cudaEventSynchronize(f1) == cudaSuccess ? 0 : NMX_ERR_CUDA;
            float ms = 0.f;
            if (!rc) cudaEventElapsedTime(&ms, f0, f1);
            cudaEventDestroy(f0);
            cudaEventDestroy(f1);
            if (rc) return rc;
            factor_extra_ms += ms;
            NMX_CUDA_TRY(cudaMemcpyAsync(x, R.xbest, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
            NMX_TRY(ir_residual(R, b, x, normA, &berr));
            prev = berr;
            use_gmres = force_gmres;
            level_steps = 0;
            since_best = 0;
        } else if (since_best >= 8) {
            break;  // no precision left to try and no progress
        }
    }
    // The best iterate is the result.
    if (!(berr <= best)) {
        NMX_CUDA_TRY(cudaMemcpyAsync(x, R.xbest, sizeof(double) * n, cudaMemcpyDeviceToDevice, st));
    }
    NMX_CUDA_TRY(cudaEventRecord(e2, st));
    NMX_CUDA_TRY(cudaEventSynchronize(e2));
    if (stats) {
        float f_ms = 0, r_ms = 0;
        cudaEventElapsedTime(&f_ms, e0, e1);
        cudaEventElapsedTime(&r_ms, e1, e2);
        stats->iterations = std::min(it, max_iter);
        stats->gmres_iterations = inner_total;
        stats->converged = best <= tol ? 1 : 0;
        stats->info = hinfo;
        stats->backward_error = best;
        stats->factor_ms = f_ms + factor_extra_ms;
        stats->refine_ms = r_ms - factor_extra_ms;
        stats->used_gmres = used_gmres ? 1 : 0;
        stats->final_precision = prec_of(R.level);
    }
    return 0;
}

}  // namespace nmx

extern "C" NMX_API int nmx_gesv_ir_f64(nmx_ctx ctx, int64_t n, const double *A, int64_t lda,
                                       const double *b, double *x, int mode, double tol,
                                       int max_iter, nmx_ir_stats *stats, void *stream) {
    return nmx::gesv_ir(ctx, n, A, lda, b, x, mode, tol, max_iter, stats, stream, false);
}

extern "C" NMX_API int nmx_posv_ir_f64(nmx_ctx ctx, int64_t n, const double *A, int64_t lda,
                                       const double *b, double *x, int mode, double tol,
                                       int max_iter, nmx_ir_stats *stats, void *stream) {
    return nmx::gesv_ir(ctx, n, A, lda, b, x, mode, tol, max_iter, stats, stream, true);
}

static int ir_reserve_entry(nmx_ctx ctx, int64_t n, int mode, bool spd) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(n >= 1 && n <= (1 << 17), 2, "n must be in 1..131072");
    const int prec = mode & 0xF;
    NMX_ARG_CHECK(prec >= NMX_IR_BF16 && prec <= NMX_IR_FP64, 3,
                  "mode must be NMX_IR_BF16/FP16/FP32/BF16X3/BF16X6/FP64 with optional flags");
    nmx::DeviceGuard g(ctx->device);
    return nmx::ir_reserve(ctx, n, nmx::level_of(prec), (mode & NMX_IR_ESCALATE) != 0, spd);
}

extern "C" NMX_API int nmx_gesv_ir_reserve(nmx_ctx ctx, int64_t n, int mode) {
    return ir_reserve_entry(ctx, n, mode, false);
}

extern "C" NMX_API int nmx_posv_ir_reserve(nmx_ctx ctx, int64_t n, int mode) {
    return ir_reserve_entry(ctx, n, mode, true);
}
