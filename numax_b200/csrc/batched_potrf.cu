// Batched uneven-size Cholesky + cho_solve (sm_100a).
//
// Replaces numax's map_blocks[step = cholesky + cholesky_solve, gpu=True]
// (numax/core/functional.mojo:691-834 driving the Array-tier bodies
// numax/linalg/_array/cholesky.mojo:26-92 and
// numax/linalg/_array/triangular.mojo:24-63), which runs one fixed-n
// problem per GPU thread out of registers.  Here each matrix of a ragged
// batch (n_i in 1..128) is staged into shared memory and factored by a whole
// CTA, blocked by 16 columns:
//
//   for each 16-column block k:
//     one warp factors the 16x16 diagonal block and forms its inverse W,
//     every thread solves rows of the panel below against W^T (a small GEMM),
//     all threads apply the symmetric trailing update in 4x4 register tiles.
//
// The right-hand sides ride along as nrhs extra rows under the matrix, so the
// forward substitution L y = b falls out of the panel solves for free; the
// back substitution L^T x = y then walks the blocks upward reusing the
// stored diagonal-block inverses.
//
// Scheduling: the plan sorts the batch by size (largest first) into buckets
// by n; each bucket is a persistent grid sized by occupancy that pulls
// matrices from an atomic work counter, so the big matrices start first and
// the small ones fill the tail.
#include <algorithm>
#include <cstring>
#include <mutex>
#include <type_traits>
#include <numeric>
#include <vector>

#include "nmx_common.cuh"

namespace nmx {

constexpr int kPotrfMaxN = 128;

// Dynamic shared memory of the batched kernels (one matrix's working set).
extern __shared__ __align__(16) unsigned char bp_smem[];
constexpr int kPotrfMaxRhs = 8;
constexpr int kDiagNB = 16;
constexpr int kPotrfStage = kDiagNB * kPotrfMaxRhs;

struct BatchedPotrfArgs {
    const int32_t *order;  // matrix indices, bucket-contiguous, largest first
    const int32_t *ns;
    const int64_t *a_off;
    const int64_t *b_off;
    const void *A;
    void *L;
    const void *B;
    void *X;
    int32_t *info;
    int nrhs;
};

// Shared-memory words (of T) one CTA needs for matrices up to nmax: the
// packed lower triangle (row i at i(i+1)/2), nrhs full rows of B^T below it,
// the reciprocals 1/l_ii of L's diagonal (nmax), and a 16 x nrhs staging
// block for the back solve.  The inverse of each
// 16x16 diagonal block is kept in place of that block once the block of L
// has been written out.
__host__ __device__ inline int potrf_smem_elems(int nmax, int nrhs) {
    return nmax * (nmax + 1) / 2 + nrhs * nmax + nmax + kPotrfStage + 2;
}

// Row of packed lower-triangle index e (e = i(i+1)/2 + j, 0 <= j <= i).
__device__ __forceinline__ int tri_row(int e) {
    int i = (int)((sqrtf(8.f * (float)e + 1.f) - 1.f) * 0.5f);
    i -= (i * (i + 1)) / 2 > e;
    i += ((i + 1) * (i + 2)) / 2 <= e;
    return i;
}

// Start of row i in the packed store: the lower triangle's rows, then the
// right-hand sides' rows (length n) below them.
__device__ __forceinline__ int prow_off(int i, int n) {
    return i < n ? (i * (i + 1)) / 2 : (n * (n + 1)) / 2 + (i - n) * n;
}

// 1/sqrt(g) from CUDA's rsqrt (faster on this chain, measured, than a
// float32 seed refined by Newton steps in float64).  A negative g gives NaN,
// as numax's sqrt of a guarded negative pivot does.
__device__ __forceinline__ double inv_sqrt(double g) { return rsqrt(g); }
__device__ __forceinline__ float inv_sqrt(float g) { return rsqrtf(g); }

// Named CTA barriers (ids 1..15; 0 is __syncthreads): a producer warp
// arrives without waiting, consumers wait for the producer and each other.
// Arrive releases and sync acquires the shared-memory writes before them.
__device__ __forceinline__ void named_barrier_arrive(int id, int nthreads) {
    asm volatile("bar.arrive %0, %1;\n" ::"r"(id), "r"(nthreads) : "memory");
}
__device__ __forceinline__ void named_barrier_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(nthreads) : "memory");
}

// Start of row k + i of the diagonal block at (k, k) in the packed store
// (k + i < n): tri(k + i) + k = tri(k) + i k + tri(i) + k.
__device__ __forceinline__ int blk_row(int tk, int k, int i) { return tk + i * k + (i * (i + 1)) / 2 + k; }

// One warp factors the kb x kb diagonal block at (k, k) in place (lane i
// holds row i in registers) with numax's Array-tier rule
// l_jj = sqrt(guard_nonzero(d, 1e-30)) (a negative d gives NaN; info records
// the first d <= 0).  Column j of L is written to shared memory as it is
// formed (the rows' packed offsets are distinct modulo 16 within a block, so
// the column store is conflict-free) and read back as broadcasts by the
// updates of the later columns; 1/l_jj goes to Dv[k + j] for the panel and
// the back solve.  At the end the block leaves for global memory as rows.
//
// The pivot chain per column is l_{j+1,j} -> d_{j+1} -> shfl -> 1/sqrt: each
// row keeps its diagonal entry in a scalar, and the next pivot's reciprocal
// square root is issued before the column's updates, which run in its
// shadow.
//
// FULL (kb == 16, every block but a matrix's last) drops the per-column
// bound tests, so the loop is one basic block.
//
// The function is not inlined, so it gets a register allocation of its own
// (inlined, it competes with the kernel's other phases and spills); the
// packed store is reached through the dynamic shared-memory symbol itself,
// which keeps its accesses in the shared window (32-bit addresses) rather
// than generic pointers.  dv_off is Dv's offset from the start of S.
//
// PIPE: after each pair of columns (2m, 2m+1) the warp arrives on named
// barrier 1 + m (nthreads = the CTA), releasing those columns to the
// warps that run the panel solve alongside (panel_trsm_pipe).
template <typename T, bool FULL, bool PIPE>
__device__ __noinline__ void potrf_diag_block(int dv_off, int n, int k, int kb_, T *Lg, int lane,
                                              int *s_info, int nthreads) {
    T *S = reinterpret_cast<T *>(bp_smem);
    T *Dv = S + dv_off;
    const int kb = FULL ? kDiagNB : kb_;
    const T floor_ = pivot_floor<T>::value;
    const int tk = (k * (k + 1)) / 2;
    // Every index into a[] below is a compile-time constant (the loops are
    // unrolled), so it stays in registers.
    T a[kDiagNB];  // strictly lower part of row `lane`
    const bool act = lane < kb;
    const int myro = blk_row(tk, k, min(lane, kb - 1));
#pragma unroll
    for (int c = 0; c < kDiagNB; ++c) a[c] = (act && c < lane) ? S[myro + c] : T(0);
    T dg = act ? S[myro + min(lane, kDiagNB - 1)] : T(1);
    int bad = 0;
    // guard_nonzero(d) is d itself for |d| >= floor (and for NaN), so the
    // reciprocal square root need not wait on the guard.
    T d = __shfl_sync(0xffffffffu, dg, 0);
    T inv = inv_sqrt(d);
    if (!(fabs(d) >= floor_)) inv = inv_sqrt(guard_nonzero(d, floor_));
#pragma unroll
    for (int j = 0; j < kDiagNB; ++j) {
        if (FULL || j < kb) {  // warp-uniform
            if (!bad && d <= T(0)) bad = k + j + 1;
            // Lane roles by selects, not branches: divergent branches here
            // cost more than the few redundant multiplies.
            const T ljj = guard_nonzero(d, floor_) * inv;
            const T lij = lane > j ? a[j] * inv : T(0);
            dg = lane == j ? ljj : dg - lij * lij;
            if (act && lane >= j) S[myro + j] = lane == j ? ljj : lij;
            if (lane == j) Dv[k + j] = inv;
            __syncwarp();
            if (FULL ? j + 1 < kDiagNB : j + 1 < kb) {
                d = __shfl_sync(0xffffffffu, dg, (j + 1) & 31);
                inv = inv_sqrt(d);
                if (!(fabs(d) >= floor_)) inv = inv_sqrt(guard_nonzero(d, floor_));
            }
            // Entries at or above a lane's diagonal are never read, so the
            // update runs unpredicated in the lane (lij is 0 on lanes <= j).
#pragma unroll
            for (int c = j + 1; c < kDiagNB; ++c)
                if (FULL || c < kb) a[c] -= lij * S[blk_row(tk, k, c) + j];
            if (PIPE && ((j & 1) || j + 1 == kb)) {
                __syncwarp();
                named_barrier_arrive(1 + (j >> 1), nthreads);
            }
        }
    }
    if (lane == 0 && bad && *s_info == 0) *s_info = bad;
    __syncwarp();
    // Two rows of the block per warp-wide store.
#pragma unroll
    for (int e = lane; e < kDiagNB * kDiagNB; e += 32) {
        const int r = e >> 4, c = e & 15;
        if (r < kb && c <= r) Lg[(int64_t)(k + r) * n + k + c] = S[blk_row(tk, k, r) + c];
    }
}

// Panel: rows r in [k+kb, R) solve x L_kk^T = S[r, k:k+kb], one thread per
// row, right-looking over the columns (x_j *= 1/l_jj, then x_i -= x_j l_ij);
// the entries of L_kk are shared-memory broadcasts.  The results are final
// rows of L (rows < n; the rows below are the right-hand sides' forward
// substitution), so they go to shared and global memory.
//
// FULL (kb == 16) drops the bound tests: loads under a run-time condition
// cannot be scheduled ahead, and that serializes the solve.
template <typename T, int NT, bool FULL>
__device__ __forceinline__ void panel_trsm(T *S, int n, int R, int k, int kb_, const T *Dv,
                                           T *Lg) {
    const int kb = FULL ? kDiagNB : kb_;
    const int tk = (k * (k + 1)) / 2;
    for (int r = k + kb + (int)threadIdx.x; r < R; r += NT) {
        const int ro = prow_off(r, n) + k;
        T x[kDiagNB];
#pragma unroll
        for (int j = 0; j < kDiagNB; ++j) x[j] = (FULL || j < kb) ? S[ro + j] : T(0);
#pragma unroll
        for (int j = 0; j < kDiagNB; ++j) {
            if (FULL || j < kb) {
                x[j] *= Dv[k + j];
#pragma unroll
                for (int i = j + 1; i < kDiagNB; ++i)
                    if (FULL || i < kb) x[i] -= x[j] * S[blk_row(tk, k, i) + j];
            }
        }
        T *lrow = Lg + (int64_t)r * n + k;
#pragma unroll
        for (int j = 0; j < kDiagNB; ++j)
            if (FULL || j < kb) {
                S[ro + j] = x[j];
                if (r < n) lrow[j] = x[j];
            }
    }
}

// Panel solve of block column k run by warps 1.. while warp 0 factors the
// diagonal block (potrf_diag_block<PIPE>): each thread takes one panel row
// (rows k+16.. of the augmented block; the thread count always covers
// them), waits on named barrier 1 + m for columns 2m, 2m+1 of L_kk, and
// applies them (x_j *= 1/l_jj, x_i -= x_j l_ij).  Every thread of warps 1..
// takes part in every barrier, with or without a row.
template <typename T, int NT, bool FULL>
__device__ __forceinline__ void panel_trsm_pipe(T *S, int n, int R, int k, int kb_, const T *Dv,
                                                T *Lg) {
    const int kb = FULL ? kDiagNB : kb_;
    const int tk = (k * (k + 1)) / 2;
    const int r = k + kb + (int)threadIdx.x - 32;
    const bool has = r < R;
    if (k + kb + (int)(threadIdx.x & ~31u) - 32 >= R) {  // no row in this warp: barriers only
#pragma unroll
        for (int j = 0; j < kDiagNB; j += 2)
            if (FULL || j < kb) named_barrier_sync(1 + (j >> 1), NT);
        return;
    }
    const int ro = prow_off(min(r, R - 1), n) + k;
    T x[kDiagNB];
#pragma unroll
    for (int j = 0; j < kDiagNB; ++j) x[j] = (has && (FULL || j < kb)) ? S[ro + j] : T(0);
#pragma unroll
    for (int j = 0; j < kDiagNB; ++j) {
        if (FULL || j < kb) {
            if ((j & 1) == 0) named_barrier_sync(1 + (j >> 1), NT);
            x[j] *= Dv[k + j];
#pragma unroll
            for (int i = j + 1; i < kDiagNB; ++i)
                if (FULL || i < kb) x[i] -= x[j] * S[blk_row(tk, k, i) + j];
        }
    }
    if (has) {
        T *lrow = Lg + (int64_t)r * n + k;
#pragma unroll
        for (int j = 0; j < kDiagNB; ++j)
            if (FULL || j < kb) {
                S[ro + j] = x[j];
                if (r < n) lrow[j] = x[j];
            }
    }
}

// ---- trailing update, CUDA-core form (float32) ---------------------------

// Flat index of a tile of the augmented trapezoid -> (tile row, tile col):
// the first TN tile rows are triangular, the rest are full TN-wide.
__device__ __forceinline__ void trap_tile(int e, int TN, int &ti, int &tj) {
    const int tri = TN * (TN + 1) / 2;
    if (e < tri) {
        ti = (int)((sqrtf(8.f * e + 1.f) - 1.f) * 0.5f);
        while (ti * (ti + 1) / 2 > e) --ti;
        while ((ti + 1) * (ti + 2) / 2 <= e) ++ti;
        tj = e - ti * (ti + 1) / 2;
    } else {
        const int e2 = e - tri;
        ti = TN + e2 / TN;
        tj = e2 - (ti - TN) * TN;
    }
}

// S[i][j] -= sum_p S[i][k+p] S[j][k+p] over rows [r0, R), cols [r0, min(i+1, n)),
// 4x4 register tiles.
template <typename T, int NT>
__device__ __forceinline__ void trailing_simt(T *S, int n, int R, int k, int kb) {
    const int tid = threadIdx.x;
    const int r0 = k + kb;
    const int TR = (int)ceil_div(R - r0, 4), TN = (int)ceil_div(n - r0, 4);
    if (TN <= 0) return;
    const int tiles = TN * (TN + 1) / 2 + (TR - TN) * TN;
    for (int e = tid; e < tiles; e += NT) {
        int ti, tj;
        trap_tile(e, TN, ti, tj);
        const int i0 = r0 + 4 * ti, j0 = r0 + 4 * tj;
        T acc[4][4];
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) acc[a][b] = T(0);
        int ir[4], jr[4];
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            ir[a] = prow_off(min(i0 + a, R - 1), n) + k;
            jr[a] = prow_off(min(j0 + a, n - 1), n) + k;
        }
        for (int p = 0; p < kb; ++p) {
            T x[4], y[4];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                x[a] = S[ir[a] + p];
                y[a] = S[jr[a] + p];
            }
#pragma unroll
            for (int a = 0; a < 4; ++a)
#pragma unroll
                for (int b = 0; b < 4; ++b) acc[a][b] += x[a] * y[b];
        }
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) {
                const int i = i0 + a, j = j0 + b;
                if (i < R && j < n && j <= i) S[ir[a] - k + j] -= acc[a][b];
            }
    }
}

// ---- panel solve and trailing update on the FP64 tensor cores ------------
// mma.sync m8n8k4 f64 (DMMA): lane l holds A[l/4][l%4], B[k=l%4][n=l/4] and
// C[l/4][2*(l%4) + {0,1}].  Rows of a fragment come from packed rows of S.

__device__ __forceinline__ void dmma_8x8x4(double &d0, double &d1, double a, double b) {
    asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
                 : "+d"(d0), "+d"(d1)
                 : "d"(a), "d"(b));
}

// One 16 x 16 tile (rows i0.., cols j0..) of the trailing update
// S[i][j] -= sum_p S[i][k+p] S[j][k+p] (p < 16), by one warp: 2 x 2 DMMA
// tiles, so each fragment loaded from shared memory feeds two DMMAs, and
// four independent accumulator chains keep the FP64 pipe busy.  On a tile
// that straddles the diagonal (i0 == j0) the block above it is skipped.
__device__ __forceinline__ void trailing_tile_dmma(double *S, int n, int R, int k, int i0, int j0) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const bool upper_skip = i0 == j0;  // rows i0..i0+7 x cols j0+8..j0+15 lie above the diagonal
    int ar[2], br[2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        ar[h] = prow_off(min(i0 + 8 * h + g, R - 1), n) + k;
        br[h] = prow_off(min(j0 + 8 * h + g, n - 1), n) + k;
    }
    double a[2][4], b[2][4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
        const int p = kk * 4 + t;
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            a[h][kk] = S[ar[h] + p];
            b[h][kk] = S[br[h] + p];
        }
    }
    double c[2][2][2] = {};
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
        dmma_8x8x4(c[0][0][0], c[0][0][1], a[0][kk], b[0][kk]);
        dmma_8x8x4(c[1][0][0], c[1][0][1], a[1][kk], b[0][kk]);
        dmma_8x8x4(c[1][1][0], c[1][1][1], a[1][kk], b[1][kk]);
        if (!upper_skip) dmma_8x8x4(c[0][1][0], c[0][1][1], a[0][kk], b[1][kk]);
    }
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int i = i0 + 8 * h + g;
        if (i >= R) continue;
        const int ro = prow_off(i, n);
#pragma unroll
        for (int hb = 0; hb < 2; ++hb) {
            const int j = j0 + 8 * hb + 2 * t;
            if (j < n && j <= i) S[ro + j] -= c[h][hb][0];
            if (j + 1 < n && j + 1 <= i) S[ro + j + 1] -= c[h][hb][1];
        }
    }
}

// Trailing update of block column k (16 wide) over the trapezoid with origin
// o (rows o..R, columns o..n, j <= i): BAND = only the 16 columns o..o+15,
// else every column from o on.  Tiles go to warps w0, w0 + nw, ...
template <bool BAND>
__device__ __forceinline__ void trailing_dmma(double *S, int n, int R, int k, int o, int w0, int nw) {
    const int warp = threadIdx.x >> 5;
    const int TR = (R - o + 15) >> 4, TN = (n - o + 15) >> 4;
    if (TN <= 0 || warp < w0) return;
    const int tiles = BAND ? TR : TN * (TN + 1) / 2 + (TR - TN) * TN;
    for (int e = warp - w0; e < tiles; e += nw) {
        int ti = e, tj = 0;
        if (!BAND) trap_tile(e, TN, ti, tj);
        trailing_tile_dmma(S, n, R, k, o + 16 * ti, o + 16 * tj);
    }
}

// ---- back substitution on the FP64 tensor cores ----------------------------

// W_b = L_bb^-1 for every 16 x 16 diagonal block, one thread per (block,
// column c): L_bb w = e_c, right-looking (w_p *= 1/l_pp, w_i -= l_ip w_p).
// Done once after the factorization, off its critical path; W_b then
// replaces L_bb in shared memory (L_bb has gone to global memory).  Needs
// NT >= 16 * ceil(n / 16), which every bucket's thread count meets.
template <int NT>
__device__ __forceinline__ void diag_inverses(double *S, int n, const double *Dv) {
    const int q = threadIdx.x;
    const int k = (q >> 4) * kDiagNB, c = q & 15;
    const int kb = min(kDiagNB, n - k);
    const bool act = k < n && c < kb;
    const int tk = (k * (k + 1)) / 2;
    double w[kDiagNB];
    if (act) {
#pragma unroll
        for (int i = 0; i < kDiagNB; ++i) w[i] = (i == c) ? 1.0 : 0.0;
#pragma unroll
        for (int p = 0; p < kDiagNB; ++p) {
            w[p] *= Dv[k + min(p, kb - 1)];
#pragma unroll
            for (int i = p + 1; i < kDiagNB; ++i) {
                // Rows past kb are clamped for the address; w stays 0 there.
                const double lip = S[blk_row(tk, k, min(i, kb - 1)) + p];
                if (i < kb) w[i] -= lip * w[p];
            }
        }
    }
    __syncthreads();
    if (act) {
#pragma unroll
        for (int i = 0; i < kDiagNB; ++i)
            if (i >= c && i < kb) S[blk_row(tk, k, i) + c] = w[i];
    }
    __syncthreads();
}

// One warp: x_blk = W^T y_blk for the block at k (16 x 16 times 16 x 8, the
// right-hand sides padded to 8 columns), 2 x 4 DMMAs.  x_blk replaces y_blk
// and goes to the staging block xb (16 x 8) for the update of the rows above.
__device__ __forceinline__ void back_block_dmma(double *S, int n, int nrhs, int k, int kb,
                                                int bro, double *xb) {
    const int lane = threadIdx.x & 31, g = lane >> 2, t = lane & 3;
    const int tk = (k * (k + 1)) / 2;
    double c[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
        const int i = kk * 4 + t;  // row of W and of y_blk
        const double bv = (g < nrhs && i < kb) ? S[bro + g * n + k + i] : 0.0;
        const int ri = blk_row(tk, k, min(i, kb - 1));
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            const int j = 8 * h + g;  // row of W^T = column of W
            const double av = (j <= i && i < kb) ? S[ri + j] : 0.0;
            dmma_8x8x4(c[h][0], c[h][1], av, bv);
        }
    }
#pragma unroll
    for (int h = 0; h < 2; ++h)
#pragma unroll
        for (int v = 0; v < 2; ++v) {
            const int j = 8 * h + g, col = 2 * t + v;
            xb[j * kPotrfMaxRhs + col] = c[h][v];  // 0 for j >= kb or col >= nrhs
            if (col < nrhs && j < kb) S[bro + col * n + k + j] = c[h][v];
        }
}

// y[0:k] -= L[k:k+16, 0:k]^T x_blk, 8-row blocks of y, one warp each,
// 4 DMMAs per block (xb rows past kb are 0).
template <int NT>
__device__ __forceinline__ void back_update_dmma(double *S, int n, int nrhs, int k, int kb,
                                                 int bro, const double *xb) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, g = lane >> 2, t = lane & 3;
    constexpr int NW = NT / 32;
    double bx[4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) bx[kk] = xb[(kk * 4 + t) * kPotrfMaxRhs + g];
    int rq[4];
#pragma unroll
    for (int kk = 0; kk < 4; ++kk) {
        const int q = min(kk * 4 + t, kb - 1);
        rq[kk] = ((k + q) * (k + q + 1)) / 2;  // start of row k + q
    }
    for (int b = warp; b < (k >> 3); b += NW) {
        const int i = 8 * b + g;
        double c0 = 0.0, c1 = 0.0;
#pragma unroll
        for (int kk = 0; kk < 4; ++kk) dmma_8x8x4(c0, c1, S[rq[kk] + i], bx[kk]);
        if (2 * t < nrhs) S[bro + (2 * t) * n + i] -= c0;
        if (2 * t + 1 < nrhs) S[bro + (2 * t + 1) * n + i] -= c1;
    }
}

// x_blk = L_kk^-T y_blk for one right-hand side (y in shared memory, rows
// k..k+kb), bottom-up: x_j = y_j / l_jj, then y_i -= l_ji x_j for i < j.
// The result replaces y and goes to column xs[0], xs[kPotrfMaxRhs], ... of
// the staging block, zero past kb.
template <typename T, bool FULL>
__device__ __forceinline__ void block_back_solve(T *y, const T *S, const T *Dv, int tk, int k,
                                                 int kb_, T *xs) {
    const int kb = FULL ? kDiagNB : kb_;
    T yv[kDiagNB];
#pragma unroll
    for (int i = 0; i < kDiagNB; ++i) yv[i] = (FULL || i < kb) ? y[min(i, kb - 1)] : T(0);
#pragma unroll
    for (int j = kDiagNB - 1; j >= 0; --j) {
        if (FULL || j < kb) {
            yv[j] *= Dv[k + j];
            const int rj = blk_row(tk, k, j);
#pragma unroll
            for (int i = 0; i < j; ++i) yv[i] -= S[rj + i] * yv[j];
        }
    }
#pragma unroll
    for (int i = 0; i < kDiagNB; ++i) {
        if (FULL || i < kb) y[i] = yv[i];
        xs[i * kPotrfMaxRhs] = (FULL || i < kb) ? yv[i] : T(0);
    }
}

// One element global -> shared without a register round trip (cp.async), so
// a thread keeps all of its staging loads in flight at once.
template <typename T>
__device__ __forceinline__ void cp_async_elem(unsigned dst, const T *src) {
    static_assert(sizeof(T) == 8 || sizeof(T) == 4, "element size");
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(dst), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

template <typename T, int NT>
__device__ void potrf_potrs_one(const BatchedPotrfArgs &args, int mi, T *S, T *Dv, T *xb,
                                int *s_info) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = NT / 32;
    const int n = args.ns[mi];
    const int nrhs = args.nrhs;
    const int R = n + nrhs;  // rows of the augmented block [A; B^T]
    const T *A = static_cast<const T *>(args.A) + args.a_off[mi];
    T *L = static_cast<T *>(args.L) + args.a_off[mi];
    const T *B = static_cast<const T *>(args.B) + args.b_off[mi];
    T *X = static_cast<T *>(args.X) + args.b_off[mi];
    if (tid == 0) *s_info = 0;

    // Stage the lower triangle (row i at i(i+1)/2) and B^T with asynchronous
    // copies, so every thread keeps all of its loads in flight.
    const int bro = (n * (n + 1)) / 2;
    {
        const unsigned sbase = (unsigned)__cvta_generic_to_shared(S);
        for (int i = warp; i < n; i += NW) {  // row i: i + 1 elements, coalesced
            const unsigned drow = sbase + (unsigned)((i * (i + 1)) / 2) * sizeof(T);
            const T *arow = A + (int64_t)i * n;
            for (int j = lane; j <= i; j += 32) cp_async_elem<T>(drow + (unsigned)j * sizeof(T), arow + j);
        }
        for (int e = tid; e < n * nrhs; e += NT) {
            const int j = e / nrhs, r = e - j * nrhs;
            cp_async_elem<T>(sbase + (unsigned)(bro + r * n + j) * sizeof(T), B + e);
        }
        cp_async_wait_all();
    }
    __syncthreads();

    const int dv_off = (int)(Dv - S);
    if constexpr (std::is_same<T, double>::value) {
        // Look-ahead: while warp 0 factors diagonal block k+16, the other
        // warps finish block k's trailing update beyond block column k+16
        // and then solve block k+16's panel column pair by column pair as
        // warp 0 releases them.  Block column k+16 itself (the band) is
        // updated first by every warp.
        auto diag_and_panel = [&](int k) {
            const int kb = min(kDiagNB, n - k);
            if (warp == 0) {
                if (kb == kDiagNB)
                    potrf_diag_block<T, true, true>(dv_off, n, k, kb, L, lane, s_info, NT);
                else
                    potrf_diag_block<T, false, true>(dv_off, n, k, kb, L, lane, s_info, NT);
            } else {
                if (k > 0 && k + kDiagNB < n)
                    trailing_dmma<false>(S, n, R, k - kDiagNB, k + kDiagNB, 1, NW - 1);
                if (kb == kDiagNB)
                    panel_trsm_pipe<T, NT, true>(S, n, R, k, kb, Dv, L);
                else
                    panel_trsm_pipe<T, NT, false>(S, n, R, k, kb, Dv, L);
            }
            __syncthreads();
        };
        diag_and_panel(0);
        for (int k = kDiagNB; k < n; k += kDiagNB) {
            trailing_dmma<true>(S, n, R, k - kDiagNB, k, 0, NW);  // the band
            __syncthreads();
            diag_and_panel(k);
        }
    } else {
        for (int k = 0; k < n; k += kDiagNB) {
            const int kb = min(kDiagNB, n - k);
            if (warp == 0) {
                if (kb == kDiagNB)
                    potrf_diag_block<T, true, false>(dv_off, n, k, kb, L, lane, s_info, NT);
                else
                    potrf_diag_block<T, false, false>(dv_off, n, k, kb, L, lane, s_info, NT);
            }
            __syncthreads();
            if (kb == kDiagNB)
                panel_trsm<T, NT, true>(S, n, R, k, kb, Dv, L);
            else
                panel_trsm<T, NT, false>(S, n, R, k, kb, Dv, L);
            __syncthreads();
            trailing_simt<T, NT>(S, n, R, k, kb);
            __syncthreads();
        }
    }

    // Rows n..n+nrhs of S now hold y^T = (L^-1 B)^T.  Back substitution
    // L^T x = y, 16-row blocks bottom-up.  FP64: the diagonal blocks are
    // inverted once (W_b), then per block x_blk = W^T y_blk and
    // y[0:k] -= L[k:k+kb, 0:k]^T x_blk are both DMMA products.
    if constexpr (std::is_same<T, double>::value) {
        if (nrhs > 0) {
            diag_inverses<NT>(S, n, Dv);
            for (int k = ((n - 1) / kDiagNB) * kDiagNB; k >= 0; k -= kDiagNB) {
                const int kb = min(kDiagNB, n - k);
                if (warp == 0) back_block_dmma(S, n, nrhs, k, kb, bro, xb);
                __syncthreads();
                back_update_dmma<NT>(S, n, nrhs, k, kb, bro, xb);
                __syncthreads();
            }
        }
    }
    // float32: x_blk solves L_kk^T x_blk = y_blk (one thread per right-hand
    // side), then y[0:k] -= L[k:k+kb, 0:k]^T x_blk (one thread per row, every
    // right-hand side at once).
    for (int k = (nrhs > 0 && !std::is_same<T, double>::value) ? ((n - 1) / kDiagNB) * kDiagNB : -1;
         k >= 0; k -= kDiagNB) {
        const int kb = min(kDiagNB, n - k);
        const int tk = (k * (k + 1)) / 2;
        for (int c = tid; c < nrhs; c += NT) {
            if (kb == kDiagNB)
                block_back_solve<T, true>(S + bro + c * n + k, S, Dv, tk, k, kb, xb + c);
            else
                block_back_solve<T, false>(S + bro + c * n + k, S, Dv, tk, k, kb, xb + c);
        }
        __syncthreads();
        for (int i = tid; i < k; i += NT) {
            T l[kDiagNB];
#pragma unroll
            for (int q = 0; q < kDiagNB; ++q) l[q] = S[blk_row(tk, k, min(q, kb - 1)) - k + i];  // xb is 0 past kb
            // The loads and multiplies run for all 4 columns of a pass (xb
            // has kPotrfMaxRhs columns; those >= nrhs are never stored):
            // loads under a run-time condition would serialize the pass.
            for (int r0 = 0; r0 < nrhs; r0 += 4) {  // 4 independent chains per pass
                T acc[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll
                for (int q = 0; q < kDiagNB; ++q)
#pragma unroll
                    for (int r = 0; r < 4; ++r) acc[r] += l[q] * xb[q * kPotrfMaxRhs + r0 + r];
#pragma unroll
                for (int r = 0; r < 4; ++r)
                    if (r0 + r < nrhs) S[bro + (r0 + r) * n + i] -= acc[r];
            }
        }
        __syncthreads();
    }

    for (int e = tid; e < n * nrhs; e += NT) {
        int j = e / nrhs, r = e - j * nrhs;
        X[e] = S[bro + r * n + j];
    }
    if (tid == 0) args.info[mi] = *s_info;
    __syncthreads();
}

// CTA shapes by bucket, each with the CTAs per SM its register budget is
// tuned for: n <= 32: 2 warps x 12; n <= 96: 4 warps x 5; n <= 128: 6 warps
// x 3 (the shared-memory limit at n = 128), which leaves 96-112 registers a
// thread in the two large shapes.  Every shape has
// threads - 32 >= n + nrhs - 16 (one panel row per thread of warps 1..) and
// threads >= 16 ceil(n / 16) (one block-inverse column per thread).
constexpr int kPotrfBigThreads = 192;
__host__ __device__ constexpr int potrf_min_blocks(int nt) {
    return nt >= 192 ? 3 : (nt >= 128 ? 5 : (nt >= 96 ? 8 : 12));
}

template <typename T, int NT>
__global__ void __launch_bounds__(NT, potrf_min_blocks(NT))
    potrf_potrs_batched_kernel(BatchedPotrfArgs args, int begin, int end, int nmax, int *counter) {
    T *S = reinterpret_cast<T *>(bp_smem);
    T *Dv = S + nmax * (nmax + 1) / 2 + args.nrhs * nmax;
    T *xb = Dv + nmax;
    __shared__ int s_item, s_info;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int item = begin + s_item;
        __syncthreads();
        if (item >= end) break;
        potrf_potrs_one<T, NT>(args, args.order[item], S, Dv, xb, &s_info);
    }
}

}  // namespace nmx

#include "batched_potrf_tile.cuh"

// ---- plan -------------------------------------------------------------------

struct nmx_batched_plan_s {
    int device = 0;
    int dtype = NMX_F64;
    int64_t count = 0;
    int nrhs = 0;
    int64_t a_elems = 0, b_elems = 0;
    void *dev = nullptr;  // one allocation for the schedule
    int32_t *d_order = nullptr, *d_n = nullptr, *d_counters = nullptr;
    int64_t *d_aoff = nullptr, *d_boff = nullptr;
    struct Bucket {
        int begin, end, nmax, threads, grid;
        size_t smem;
    };
    std::vector<Bucket> buckets;
    // CUDA graph of one run, for the buffers in graph_key (A, L, B, X, info).
    cudaGraphExec_t graph = nullptr;
    const void *graph_key[5] = {nullptr, nullptr, nullptr, nullptr, nullptr};
};

namespace nmx {

static const int kBucketEdges[] = {32, 64, 96, 128};

static int potrf_threads_for(int nmax) {
    return nmax <= 32 ? 64 : (nmax <= 96 ? 128 : kPotrfBigThreads);
}

// CTA shapes 1032, 1064, 1128 and 1256 (1000 + threads) select the 8 x 8
// DMMA tile kernel with 1, 2, 4 or 8 warps per matrix (FP64 arithmetic for
// both element types, batched_potrf_tile.cuh); 64, 96, 128 and 192
// potrf_potrs_batched_kernel.
static const int kAllShapes[] = {64, 96, 128, 192, kTileShapeBase + 32, kTileShapeBase + 64,
                                 kTileShapeBase + 128, kTileShapeBase + 256};

// Dynamic shared memory of a CTA shape for a bucket of matrices up to nmax.
template <typename T>
static size_t shape_smem(int threads, int nmax, int nrhs) {
    if (is_tile_shape(threads)) return sizeof(double) * (size_t)tile_smem_doubles(nmax, nrhs);
    return sizeof(T) * (size_t)potrf_smem_elems(nmax, nrhs);
}

template <typename T>
static int launch_bucket(const BatchedPotrfArgs &args, const nmx_batched_plan_s::Bucket &b,
                         int *counter, cudaStream_t st) {
    switch (b.threads) {
#define NMX_CASE(NTV)                                                                        \
    case NTV:                                                                                \
        potrf_potrs_batched_kernel<T, NTV><<<b.grid, NTV, b.smem, st>>>(args, b.begin, b.end, \
                                                                        b.nmax, counter);    \
        break;
        NMX_CASE(64)
        NMX_CASE(96)
        NMX_CASE(128)
        NMX_CASE(192)
#undef NMX_CASE
#define NMX_TCASE(WPM)                                                                   \
    case kTileShapeBase + 32 * WPM:                                                       \
        potrf_tile_batched_kernel<WPM, T><<<b.grid, 32 * WPM, b.smem, st>>>(args, b.begin, \
                                                                          b.end, b.nmax,  \
                                                                          counter);       \
        break;
        NMX_TCASE(1)
        NMX_TCASE(2)
        NMX_TCASE(4)
        NMX_TCASE(8)
#undef NMX_TCASE
        default:
            set_error("unsupported thread count %d", b.threads);
            return NMX_ERR_INTERNAL;
    }
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

// Let a kernel use all the opt-in shared memory not taken by its static
// shared variables (the largest bucket's size decides the launch).
template <typename K>
static cudaError_t set_max_dynamic_smem(K kernel, nmx_ctx ctx) {
    cudaFuncAttributes fa;
    cudaError_t e = cudaFuncGetAttributes(&fa, kernel);
    if (e != cudaSuccess) return e;
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(ctx->smem_optin - fa.sharedSizeBytes));
}

// Whether a CTA of `threads` covers a bucket of matrices up to nmax with nrhs
// right-hand sides (one panel row per thread of warps 1.., one
// block-inverse column per thread).
static bool shape_covers(int threads, int nmax, int nrhs) {
    return threads - 32 >= nmax + nrhs - std::min(nmax, kDiagNB) &&
           threads >= kDiagNB * (int)ceil_div(nmax, kDiagNB);
}

// CTAs per SM of the kernel with `threads` at `smem` bytes (0: does not fit).
template <typename T>
static int shape_occupancy(nmx_ctx ctx, int threads, size_t smem, int *per_sm) {
    *per_sm = 0;
    switch (threads) {
#define NMX_OCC(NTV)                                                                           \
    case NTV:                                                                                  \
        NMX_CUDA_TRY(set_max_dynamic_smem(potrf_potrs_batched_kernel<T, NTV>, ctx));        \
        NMX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(                            \
            per_sm, potrf_potrs_batched_kernel<T, NTV>, NTV, smem));                           \
        break;
        NMX_OCC(64)
        NMX_OCC(96)
        NMX_OCC(128)
        NMX_OCC(192)
#undef NMX_OCC
#define NMX_TOCC(WPM)                                                                   \
    case kTileShapeBase + 32 * WPM:                                                      \
        NMX_CUDA_TRY(set_max_dynamic_smem(potrf_tile_batched_kernel<WPM, T>, ctx));      \
        NMX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(                      \
            per_sm, potrf_tile_batched_kernel<WPM, T>, 32 * WPM, smem));                 \
        break;
        NMX_TOCC(1)
        NMX_TOCC(2)
        NMX_TOCC(4)
        NMX_TOCC(8)
#undef NMX_TOCC
        default:
            break;
    }
    return 0;
}

// Default CTA shape of a bucket: the tile kernel with 1 warp per matrix up
// to n = 64, 2 up to 96 and 4 up to 128 (the fastest shapes on a B200 for
// n ~ U[8, 128] with 4 right-hand sides, FP64 and FP32 alike).
template <typename T>
static int default_shape(int nmax) {
    return kTileShapeBase + 32 * (nmax <= 64 ? 1 : (nmax <= 96 ? 2 : 4));
}

template <typename T>
static int configure_buckets(nmx_ctx ctx, nmx_batched_plan_s *p) {
    for (auto &b : p->buckets) {
        b.threads = default_shape<T>(b.nmax);
        if (!is_tile_shape(b.threads) && !shape_covers(b.threads, b.nmax, p->nrhs)) {
            set_error("internal: %d threads cannot cover n=%d with %d right-hand sides", b.threads,
                      b.nmax, p->nrhs);
            return NMX_ERR_INTERNAL;
        }
        b.smem = shape_smem<T>(b.threads, b.nmax, p->nrhs);
        if (b.smem + 64 > ctx->smem_optin) {
            set_error("bucket nmax=%d needs %zu B of shared memory (> %zu)", b.nmax, b.smem,
                      ctx->smem_optin);
            return NMX_ERR_UNSUPPORTED;
        }
        int per_sm = 0;
        int rc = shape_occupancy<T>(ctx, b.threads, b.smem, &per_sm);
        if (rc) return rc;
        if (per_sm < 1) {
            set_error("bucket nmax=%d does not fit on an SM (smem %zu)", b.nmax, b.smem);
            return NMX_ERR_UNSUPPORTED;
        }
        int64_t work = b.end - b.begin;
        b.grid = (int)std::min<int64_t>(work, (int64_t)per_sm * ctx->sm_count);
    }
    return 0;
}

template <typename T>
static int run_potrf_potrs(nmx_ctx ctx, nmx_batched_plan plan, const T *A, T *L, const T *B,
                           T *X, int32_t *info, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(plan != nullptr, 2, "plan is NULL");
    NMX_ARG_CHECK(plan->dtype == (sizeof(T) == 8 ? NMX_F64 : NMX_F32), 2,
                  "plan was built for the other dtype");
    NMX_ARG_CHECK(A != nullptr || plan->count == 0, 3, "A is NULL");
    NMX_ARG_CHECK(L != nullptr || plan->count == 0, 4, "L is NULL");
    NMX_ARG_CHECK(B != nullptr || plan->nrhs == 0 || plan->count == 0, 5, "B is NULL");
    NMX_ARG_CHECK(X != nullptr || plan->nrhs == 0 || plan->count == 0, 6, "X is NULL");
    NMX_ARG_CHECK(info != nullptr || plan->count == 0, 7, "info is NULL");
    if (plan->count == 0) return 0;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    BatchedPotrfArgs args{plan->d_order, plan->d_n, plan->d_aoff, plan->d_boff, A,
                          L,             B,         X,            info,         plan->nrhs};
    NMX_CUDA_TRY(cudaMemsetAsync(plan->d_counters, 0, sizeof(int32_t) * plan->buckets.size(), st));
    for (size_t bi = 0; bi < plan->buckets.size(); ++bi) {
        int rc = launch_bucket<T>(args, plan->buckets[bi], plan->d_counters + bi, st);
        if (rc) return rc;
    }
    return 0;
}

// Time every covering CTA shape of every bucket on these buffers (each
// bucket's kernel alone, best of `reps` runs, CUDA events on `st`) and keep
// the fastest.  Every run computes the full bucket, so the outputs hold a
// valid result afterwards.
template <typename T>
static int autotune(nmx_ctx ctx, nmx_batched_plan plan, const T *A, T *L, const T *B, T *X,
                    int32_t *info, int reps, cudaStream_t st) {
    BatchedPotrfArgs args{plan->d_order, plan->d_n, plan->d_aoff, plan->d_boff, A,
                          L,             B,         X,            info,         plan->nrhs};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    NMX_CUDA_TRY(cudaEventCreate(&e0));
    cudaError_t ce = cudaEventCreate(&e1);
    if (ce != cudaSuccess) {
        cudaEventDestroy(e0);
        NMX_CUDA_TRY(ce);
    }
    int rc = 0;
    for (size_t bi = 0; bi < plan->buckets.size() && !rc; ++bi) {
        auto best = plan->buckets[bi];
        float best_ms = 3.4e38f;
        for (int threads : kAllShapes) {
            auto cand = plan->buckets[bi];
            if (!is_tile_shape(threads) && !shape_covers(threads, cand.nmax, plan->nrhs)) {
                continue;
            }
            cand.threads = threads;
            cand.smem = shape_smem<T>(threads, cand.nmax, plan->nrhs);
            int per_sm = 0;
            rc = shape_occupancy<T>(ctx, threads, cand.smem, &per_sm);
            if (rc) break;
            if (per_sm < 1) continue;
            cand.grid = (int)std::min<int64_t>(cand.end - cand.begin, (int64_t)per_sm * ctx->sm_count);
            float ms = 3.4e38f;
            for (int r = 0; r < std::max(1, reps) && !rc; ++r) {
                if (cudaMemsetAsync(plan->d_counters + bi, 0, sizeof(int32_t), st) != cudaSuccess ||
                    cudaEventRecord(e0, st) != cudaSuccess) {
                    set_error("autotune: %s", cudaGetErrorString(cudaGetLastError()));
                    rc = NMX_ERR_CUDA;
                    break;
                }
                rc = launch_bucket<T>(args, cand, plan->d_counters + bi, st);
                float t = 0.f;
                if (!rc && (cudaEventRecord(e1, st) != cudaSuccess ||
                            cudaEventSynchronize(e1) != cudaSuccess ||
                            cudaEventElapsedTime(&t, e0, e1) != cudaSuccess)) {
                    set_error("autotune: %s", cudaGetErrorString(cudaGetLastError()));
                    rc = NMX_ERR_CUDA;
                }
                ms = std::min(ms, t);
            }
            if (rc) break;
            if (ms < best_ms) {
                best_ms = ms;
                best = cand;
            }
        }
        plan->buckets[bi] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (plan->graph) {  // the captured shapes are stale
        cudaGraphExecDestroy(plan->graph);
        plan->graph = nullptr;
    }
    return rc;
}

// Run the plan through a CUDA graph of its launches (counter reset and one
// persistent kernel per bucket), captured on an internal stream the first
// time these buffers are seen and replayed on `stream` after that.
template <typename T>
static int run_graph(nmx_ctx ctx, nmx_batched_plan plan, const T *A, T *L, const T *B, T *X,
                     int32_t *info, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(plan != nullptr, 2, "plan is NULL");
    if (plan->count == 0) return 0;
    DeviceGuard g(ctx->device);
    const void *key[5] = {A, L, B, X, info};
    if (!plan->graph || !std::equal(key, key + 5, plan->graph_key)) {
        if (plan->graph) {
            cudaGraphExecDestroy(plan->graph);
            plan->graph = nullptr;
        }
        cudaStream_t cs = nullptr;
        NMX_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t graph = nullptr;
        int rc = 0;
        if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            set_error("graph capture: %s", cudaGetErrorString(cudaGetLastError()));
            rc = NMX_ERR_CUDA;
        } else {
            rc = run_potrf_potrs<T>(ctx, plan, A, L, B, X, info, cs);
            cudaError_t e = cudaStreamEndCapture(cs, &graph);
            if (!rc && e != cudaSuccess) {
                set_error("graph capture: %s", cudaGetErrorString(e));
                rc = NMX_ERR_CUDA;
            }
        }
        if (!rc && cudaGraphInstantiate(&plan->graph, graph, 0) != cudaSuccess) {
            set_error("graph instantiate: %s", cudaGetErrorString(cudaGetLastError()));
            plan->graph = nullptr;
            rc = NMX_ERR_CUDA;
        }
        if (graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cs);
        if (rc) return rc;
        std::copy(key, key + 5, plan->graph_key);
    }
    NMX_CUDA_TRY(cudaGraphLaunch(plan->graph, static_cast<cudaStream_t>(stream)));
    return 0;
}

}  // namespace nmx

extern "C" {

int nmx_potrf_potrs_batched_plan(nmx_ctx ctx, int dtype, int64_t count, const int32_t *n_host,
                                 int nrhs, nmx_batched_plan *out) {
    using namespace nmx;
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(dtype == NMX_F32 || dtype == NMX_F64, 2, "dtype must be NMX_F32 or NMX_F64");
    NMX_ARG_CHECK(count >= 0 && count < (int64_t(1) << 31), 3, "count out of range");
    NMX_ARG_CHECK(n_host != nullptr || count == 0, 4, "n_host is NULL");
    NMX_ARG_CHECK(nrhs >= 0 && nrhs <= kPotrfMaxRhs, 5, "nrhs must be in 0..8");
    NMX_ARG_CHECK(out != nullptr, 6, "out is NULL");
    for (int64_t i = 0; i < count; ++i)
        NMX_ARG_CHECK(n_host[i] >= 1 && n_host[i] <= kPotrfMaxN, 4, "every n_i must be in 1..128");
    *out = nullptr;
    DeviceGuard g(ctx->device);
    auto *p = new (std::nothrow) nmx_batched_plan_s();
    if (!p) return NMX_ERR_ALLOC;
    p->device = ctx->device;
    p->dtype = dtype;
    p->count = count;
    p->nrhs = nrhs;
    std::vector<int64_t> aoff(count), boff(count);
    int64_t a = 0, b = 0;
    for (int64_t i = 0; i < count; ++i) {
        aoff[i] = a;
        boff[i] = b;
        a += (int64_t)n_host[i] * n_host[i];
        b += (int64_t)n_host[i] * nrhs;
    }
    p->a_elems = a;
    p->b_elems = b;
    // Bucket-contiguous order, largest n first inside each bucket, buckets
    // from the largest down (longest-processing-time first).
    std::vector<int32_t> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t x, int32_t y) { return n_host[x] > n_host[y]; });
    int64_t pos = 0;
    for (int e = 3; e >= 0 && pos < count; --e) {
        int lo = e == 0 ? 0 : kBucketEdges[e - 1];
        int64_t begin = pos;
        while (pos < count && n_host[order[pos]] > lo) ++pos;
        if (pos > begin)
            p->buckets.push_back({(int)begin, (int)pos, n_host[order[begin]], 0, 0, 0});
    }
    size_t nb = p->buckets.size();
    size_t bytes = sizeof(int32_t) * (2 * count + nb + 1) + sizeof(int64_t) * (2 * count) + 64;
    cudaError_t e = cudaMalloc(&p->dev, bytes);
    if (e != cudaSuccess) {
        delete p;
        set_error("plan cudaMalloc: %s", cudaGetErrorString(e));
        return NMX_ERR_ALLOC;
    }
    char *base = static_cast<char *>(p->dev);
    p->d_aoff = reinterpret_cast<int64_t *>(base);
    p->d_boff = p->d_aoff + count;
    p->d_order = reinterpret_cast<int32_t *>(p->d_boff + count);
    p->d_n = p->d_order + count;
    p->d_counters = p->d_n + count;
    int rc = 0;
    if (count) {
        if (cudaMemcpy(p->d_aoff, aoff.data(), sizeof(int64_t) * count, cudaMemcpyHostToDevice) ||
            cudaMemcpy(p->d_boff, boff.data(), sizeof(int64_t) * count, cudaMemcpyHostToDevice) ||
            cudaMemcpy(p->d_order, order.data(), sizeof(int32_t) * count, cudaMemcpyHostToDevice) ||
            cudaMemcpy(p->d_n, n_host, sizeof(int32_t) * count, cudaMemcpyHostToDevice)) {
            set_error("plan upload failed");
            rc = NMX_ERR_CUDA;
        }
    }
    if (!rc) rc = dtype == NMX_F64 ? configure_buckets<double>(ctx, p) : configure_buckets<float>(ctx, p);
    if (rc) {
        cudaFree(p->dev);
        delete p;
        return rc;
    }
    *out = p;
    return 0;
}

int nmx_batched_plan_destroy(nmx_batched_plan plan) {
    if (!plan) return 0;
    nmx::DeviceGuard g(plan->device);
    if (plan->graph) cudaGraphExecDestroy(plan->graph);
    if (plan->dev) cudaFree(plan->dev);
    delete plan;
    return 0;
}

int nmx_batched_plan_sizes(nmx_batched_plan plan, int64_t *a_elems, int64_t *b_elems) {
    NMX_ARG_CHECK(plan != nullptr, 1, "plan is NULL");
    if (a_elems) *a_elems = plan->a_elems;
    if (b_elems) *b_elems = plan->b_elems;
    return 0;
}

int nmx_potrf_potrs_batched_f64(nmx_ctx ctx, nmx_batched_plan plan, const double *A, double *L,
                                const double *B, double *X, int32_t *info, void *stream) {
    return nmx::run_potrf_potrs<double>(ctx, plan, A, L, B, X, info, stream);
}

int nmx_potrf_potrs_batched_f32(nmx_ctx ctx, nmx_batched_plan plan, const float *A, float *L,
                                const float *B, float *X, int32_t *info, void *stream) {
    return nmx::run_potrf_potrs<float>(ctx, plan, A, L, B, X, info, stream);
}

int nmx_batched_plan_autotune(nmx_ctx ctx, nmx_batched_plan plan, const void *A, void *L,
                              const void *B, void *X, int32_t *info, int reps, void *stream) {
    using namespace nmx;
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(plan != nullptr, 2, "plan is NULL");
    NMX_ARG_CHECK(A != nullptr || plan->count == 0, 3, "A is NULL");
    NMX_ARG_CHECK(L != nullptr || plan->count == 0, 4, "L is NULL");
    NMX_ARG_CHECK(B != nullptr || plan->nrhs == 0 || plan->count == 0, 5, "B is NULL");
    NMX_ARG_CHECK(X != nullptr || plan->nrhs == 0 || plan->count == 0, 6, "X is NULL");
    NMX_ARG_CHECK(info != nullptr || plan->count == 0, 7, "info is NULL");
    NMX_ARG_CHECK(reps >= 1 && reps <= 100, 8, "reps must be in 1..100");
    if (plan->count == 0) return 0;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    if (plan->dtype == NMX_F64)
        return autotune<double>(ctx, plan, static_cast<const double *>(A), static_cast<double *>(L),
                                static_cast<const double *>(B), static_cast<double *>(X), info,
                                reps, st);
    return autotune<float>(ctx, plan, static_cast<const float *>(A), static_cast<float *>(L),
                           static_cast<const float *>(B), static_cast<float *>(X), info, reps, st);
}

int nmx_batched_plan_schedule(nmx_batched_plan plan, int32_t *nmax, int32_t *threads,
                              int32_t *ctas, int max_buckets, int32_t *nbuckets) {
    NMX_ARG_CHECK(plan != nullptr, 1, "plan is NULL");
    NMX_ARG_CHECK(max_buckets >= 0, 5, "max_buckets < 0");
    const int nb = (int)plan->buckets.size();
    for (int i = 0; i < nb && i < max_buckets; ++i) {
        if (nmax) nmax[i] = plan->buckets[i].nmax;
        if (threads) threads[i] = plan->buckets[i].threads;
        if (ctas) ctas[i] = plan->buckets[i].grid;
    }
    if (nbuckets) *nbuckets = nb;
    return 0;
}

int nmx_batched_partition(int64_t count, const int32_t *n_host, int nrhs, int ndev,
                          int32_t *dev_of, double *cost_per_dev) {
    using namespace nmx;
    NMX_ARG_CHECK(count >= 0 && count < (int64_t(1) << 31), 1, "count out of range");
    NMX_ARG_CHECK(n_host != nullptr || count == 0, 2, "n_host is NULL");
    NMX_ARG_CHECK(nrhs >= 0 && nrhs <= kPotrfMaxRhs, 3, "nrhs must be in 0..8");
    NMX_ARG_CHECK(ndev >= 1 && ndev <= 1024, 4, "ndev must be in 1..1024");
    NMX_ARG_CHECK(dev_of != nullptr || count == 0, 5, "dev_of is NULL");
    for (int64_t i = 0; i < count; ++i)
        NMX_ARG_CHECK(n_host[i] >= 1 && n_host[i] <= kPotrfMaxN, 2, "every n_i must be in 1..128");
    // Cost of one matrix: its flops (n^3/3 for the factor, 2 nrhs n^2 for the
    // solves) plus its bytes (n^2 read and written, 8 bytes each) weighted as
    // flops at the FP64 / HBM balance of the part (about 6 flops a byte).
    auto cost = [&](int n) {
        const double d = n;
        return d * d * d / 3.0 + 2.0 * nrhs * d * d + 6.0 * 16.0 * d * d;
    };
    // Longest processing time first: matrices by cost descending (index
    // ascending among equals, so the split is deterministic), each to the
    // least-loaded device (lowest index among equals).
    std::vector<int32_t> order((size_t)count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t a, int32_t b) { return n_host[a] > n_host[b]; });
    std::vector<double> load((size_t)ndev, 0.0);
    // A min-heap of (load, device) would be O(log ndev) per matrix; ndev is
    // small, so a linear scan keeps the tie-breaking obvious.
    for (int32_t i : order) {
        int best = 0;
        for (int d = 1; d < ndev; ++d)
            if (load[d] < load[best]) best = d;
        dev_of[i] = best;
        load[best] += cost(n_host[i]);
    }
    if (cost_per_dev)
        for (int d = 0; d < ndev; ++d) cost_per_dev[d] = load[d];
    return 0;
}

int nmx_batched_plan_set_shape(nmx_ctx ctx, nmx_batched_plan plan, int bucket, int threads) {
    using namespace nmx;
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(plan != nullptr, 2, "plan is NULL");
    NMX_ARG_CHECK(bucket >= -1 && bucket < (int)plan->buckets.size(), 3,
                  "bucket must be -1 (all) or a bucket index");
    NMX_ARG_CHECK(threads == 64 || threads == 96 || threads == 128 || threads == 192 ||
                      is_tile_shape(threads),
                  4, "threads must be 64, 96, 128, 192, or 1032, 1064, 1128, 1256 (the tile kernel)");
    DeviceGuard g(ctx->device);
    for (int bi = 0; bi < (int)plan->buckets.size(); ++bi) {
        if (bucket >= 0 && bi != bucket) continue;
        auto &b = plan->buckets[bi];
        NMX_ARG_CHECK(is_tile_shape(threads) || shape_covers(threads, b.nmax, plan->nrhs), 4,
                      "that CTA shape cannot cover this bucket's sizes");
        const size_t smem = plan->dtype == NMX_F64 ? shape_smem<double>(threads, b.nmax, plan->nrhs)
                                                   : shape_smem<float>(threads, b.nmax, plan->nrhs);
        int per_sm = 0;
        const int rc = plan->dtype == NMX_F64 ? shape_occupancy<double>(ctx, threads, smem, &per_sm)
                                              : shape_occupancy<float>(ctx, threads, smem, &per_sm);
        if (rc) return rc;
        if (per_sm < 1) {
            set_error("that CTA shape does not fit an SM for n up to %d", b.nmax);
            return NMX_ERR_UNSUPPORTED;
        }
        b.threads = threads;
        b.smem = smem;
        b.grid = (int)std::min<int64_t>(b.end - b.begin, (int64_t)per_sm * ctx->sm_count);
    }
    if (plan->graph) {  // the captured shapes are stale
        cudaGraphExecDestroy(plan->graph);
        plan->graph = nullptr;
    }
    return 0;
}

int nmx_potrf_potrs_batched_graph_f64(nmx_ctx ctx, nmx_batched_plan plan, const double *A,
                                      double *L, const double *B, double *X, int32_t *info,
                                      void *stream) {
    return nmx::run_graph<double>(ctx, plan, A, L, B, X, info, stream);
}

int nmx_potrf_potrs_batched_graph_f32(nmx_ctx ctx, nmx_batched_plan plan, const float *A, float *L,
                                      const float *B, float *X, int32_t *info, void *stream) {
    return nmx::run_graph<float>(ctx, plan, A, L, B, X, info, stream);
}

}  // extern "C"

// ---- allocation-free entry point --------------------------------------------
//
// For callers that cannot allocate device memory (a host runtime whose
// allocator owns all of HBM, or code running inside another framework's
// memory pool): the same kernel as the plan path, with
// its schedule -- matrix sizes, size-sorted order, element offsets and the
// work counter -- held in a fixed file-scope device array instead of a plan's
// cudaMalloc'd buffer.  The array is sized for kNoAllocMaxCount matrices
// (about 1.5 MB) and lives on every GPU that loads the library until exit.

namespace nmx {

constexpr int64_t kNoAllocMaxCount = 65536;
constexpr size_t kNoAllocScratchBytes = (size_t)kNoAllocMaxCount * (4 + 4 + 8 + 8) + 256;

// Layout: int32 n[max] | int32 order[max] | int64 a_off[max] | int64 b_off[max] | int32 counter.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

struct NoAllocViews {
    int32_t *n, *order;
    int64_t *a_off, *b_off;
    int32_t *counter;
};

__host__ __device__ inline NoAllocViews noalloc_views(unsigned char *base) {
    NoAllocViews v;
    v.n = reinterpret_cast<int32_t *>(base);
    v.order = v.n + kNoAllocMaxCount;
    v.a_off = reinterpret_cast<int64_t *>(v.order + kNoAllocMaxCount);
    v.b_off = v.a_off + kNoAllocMaxCount;
    v.counter = reinterpret_cast<int32_t *>(v.b_off + kNoAllocMaxCount);
    return v;
}

// One CTA: element offsets (exclusive prefix sums of n^2 and n*nrhs), the
// order sorted by n descending (counting sort), and a zeroed work counter.
constexpr int kSchedThreads = 1024;
__global__ void __launch_bounds__(kSchedThreads) noalloc_schedule_kernel(unsigned char *scratch,
                                                                         int count, int nrhs) {
    NoAllocViews v = noalloc_views(scratch);
    __shared__ int64_t part_a[kSchedThreads], part_b[kSchedThreads];
    __shared__ int hist[kPotrfMaxN + 1], start[kPotrfMaxN + 1];
    const int t = threadIdx.x;
    const int per = (count + kSchedThreads - 1) / kSchedThreads;
    const int lo = min(count, t * per), hi = min(count, lo + per);
    int64_t sa = 0, sb = 0;
    for (int i = lo; i < hi; ++i) {
        int64_t n = v.n[i];
        sa += n * n;
        sb += n * nrhs;
    }
    part_a[t] = sa;
    part_b[t] = sb;
    for (int i = t; i <= kPotrfMaxN; i += kSchedThreads) hist[i] = 0;
    __syncthreads();
    if (t == 0) {
        int64_t ra = 0, rb = 0;
        for (int i = 0; i < kSchedThreads; ++i) {
            int64_t a = part_a[i], b = part_b[i];
            part_a[i] = ra;
            part_b[i] = rb;
            ra += a;
            rb += b;
        }
    }
    __syncthreads();
    sa = part_a[t];
    sb = part_b[t];
    for (int i = lo; i < hi; ++i) {
        int64_t n = v.n[i];
        v.a_off[i] = sa;
        v.b_off[i] = sb;
        sa += n * n;
        sb += n * nrhs;
        atomicAdd(&hist[n], 1);
    }
    __syncthreads();
    if (t == 0) {
        int pos = 0;
        for (int n = kPotrfMaxN; n >= 1; --n) {
            start[n] = pos;
            pos += hist[n];
        }
        *v.counter = 0;
    }
    __syncthreads();
    for (int i = lo; i < hi; ++i) v.order[atomicAdd(&start[v.n[i]], 1)] = i;
}

struct NoAllocDevice {
    bool ready = false;
    unsigned char *scratch = nullptr;  // device address of g_noalloc_scratch
    int sm_count = 0;
    int per_sm[2] = {0, 0};  // potrf_potrs_batched_kernel<T, kPotrfBigThreads> at nmax=128, nrhs=8
};
static NoAllocDevice g_noalloc_dev[64];
static std::mutex g_noalloc_mu;

// Per-device set-up, run by the first call on each device with that device
// current: resolve the array's device address (host code cannot use the
// symbol itself) and configure the kernel.
template <typename T>
static int noalloc_setup(nmx_ctx ctx, NoAllocDevice **out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    if (ctx->device < 0 || ctx->device >= 64) {
        set_error("device ordinal %d out of range", ctx->device);
        return NMX_ERR_UNSUPPORTED;
    }
    NoAllocDevice &d = g_noalloc_dev[ctx->device];
    const int ti = sizeof(T) == 8 ? 0 : 1;
    if (!d.ready) {
        void *ptr = nullptr;
        NMX_CUDA_TRY(cudaGetSymbolAddress(&ptr, g_noalloc_scratch));
        d.scratch = static_cast<unsigned char *>(ptr);
        d.sm_count = ctx->sm_count;
        d.ready = true;
    }
    if (d.per_sm[ti] == 0) {
        auto kern = potrf_potrs_batched_kernel<T, kPotrfBigThreads>;
        NMX_CUDA_TRY(set_max_dynamic_smem(kern, ctx));
        size_t smem = sizeof(T) * (size_t)potrf_smem_elems(kPotrfMaxN, kPotrfMaxRhs);
        int per_sm = 0;
        NMX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kPotrfBigThreads, smem));
        if (per_sm < 1) {
            set_error("allocation-free kernel does not fit an SM");
            return NMX_ERR_UNSUPPORTED;
        }
        d.per_sm[ti] = per_sm;
    }
    *out = &d;
    return 0;
}

template <typename T>
static int run_noalloc(nmx_ctx ctx, int64_t count, const int32_t *n_host, int nrhs, const T *A,
                       T *L, const T *B, T *X, int32_t *info, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(count >= 0, 2, "count < 0");
    if (count > kNoAllocMaxCount) {
        set_error("argument 2: count %lld exceeds the allocation-free limit of %lld matrices "
                  "(use the plan entry points for larger batches)",
                  (long long)count, (long long)kNoAllocMaxCount);
        return -2;
    }
    NMX_ARG_CHECK(n_host != nullptr || count == 0, 3, "n_host is NULL");
    NMX_ARG_CHECK(nrhs >= 0 && nrhs <= kPotrfMaxRhs, 4, "nrhs must be in 0..8");
    NMX_ARG_CHECK(A != nullptr || count == 0, 5, "A is NULL");
    NMX_ARG_CHECK(L != nullptr || count == 0, 6, "L is NULL");
    NMX_ARG_CHECK(B != nullptr || nrhs == 0 || count == 0, 7, "B is NULL");
    NMX_ARG_CHECK(X != nullptr || nrhs == 0 || count == 0, 8, "X is NULL");
    NMX_ARG_CHECK(info != nullptr || count == 0, 9, "info is NULL");
    int nmax = 1;
    for (int64_t i = 0; i < count; ++i) {
        NMX_ARG_CHECK(n_host[i] >= 1 && n_host[i] <= kPotrfMaxN, 3, "every n_i must be in 1..128");
        nmax = std::max(nmax, (int)n_host[i]);
    }
    if (count == 0) return 0;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // The sizes are checked on the host and the launch is sized for them at
    // call time, so a captured call would replay with whatever n_host holds
    // later, unchecked.  Refuse capture instead.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    NMX_CUDA_TRY(cudaStreamIsCapturing(st, &cap));
    if (cap != cudaStreamCaptureStatusNone) {
        set_error("the allocation-free entry point checks n_host on the host at each call and "
                  "cannot run while its stream is being captured");
        return NMX_ERR_UNSUPPORTED;
    }
    NoAllocDevice *d = nullptr;
    int rc = noalloc_setup<T>(ctx, &d);
    if (rc) return rc;
    NoAllocViews v = noalloc_views(d->scratch);
    NMX_CUDA_TRY(cudaMemcpyAsync(v.n, n_host, sizeof(int32_t) * count, cudaMemcpyHostToDevice, st));
    noalloc_schedule_kernel<<<1, kSchedThreads, 0, st>>>(d->scratch, (int)count, nrhs);
    NMX_CUDA_TRY(cudaGetLastError());
    BatchedPotrfArgs args{v.order, v.n, v.a_off, v.b_off, A, L, B, X, info, nrhs};
    const size_t smem = sizeof(T) * (size_t)potrf_smem_elems(nmax, nrhs);
    const int grid = (int)std::min<int64_t>(count, (int64_t)d->per_sm[sizeof(T) == 8 ? 0 : 1] *
                                                       d->sm_count);
    potrf_potrs_batched_kernel<T, kPotrfBigThreads><<<grid, kPotrfBigThreads, smem, st>>>(args, 0, (int)count, nmax,
                                                                v.counter);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

}  // namespace nmx

extern "C" NMX_API int nmx_potrf_potrs_batched_noalloc_f64(nmx_ctx ctx, int64_t count,
                                                           const int32_t *n_host, int nrhs,
                                                           const double *A, double *L,
                                                           const double *B, double *X,
                                                           int32_t *info, void *stream) {
    return nmx::run_noalloc<double>(ctx, count, n_host, nrhs, A, L, B, X, info, stream);
}
