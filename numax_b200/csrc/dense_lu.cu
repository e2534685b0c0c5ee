// Dense LU with partial pivoting and the LU solve (sm_100a), row-major.
//
// numax's lu_factor (numax/linalg/lu.mojo:454-701) is right-looking and
// blocked (block 16 on a device) with a recursive panel getrf2
// (numax/linalg/panel.mojo:445-586) whose leaves are a single-CTA
// getrf_panel (numax/linalg/panel.mojo:289-431); its cubic term is MAX's
// matmul.  Here the recursion is taken all the way up -- getrf2 over the
// whole matrix -- so every cubic term is one large GEMM, and the leaves
// (32 columns) are factored by a cooperative kernel that spreads the panel's
// rows over every SM:
//
//   per column: each CTA finds its local max |a| (first maximum, lower row
//   on ties: numax's pivot rule), publishes the candidate row, one grid-wide
//   barrier, every CTA picks the same winner, the two owners exchange rows,
//   every CTA scales and rank-1 updates its own rows.
//
// One barrier per column; the published rows are double-buffered by column
// parity so a fast CTA never overwrites what a slow one still reads.
// Interchanges are recorded LAPACK-style (pivots[j] = row swapped with j,
// 0-based) and applied across the full width, as numax does: inside the leaf
// to the leaf's columns, then by a laswp kernel to every other column.
#include <cooperative_groups.h>

#include <algorithm>

#include "calu.cuh"
#include "dense_common.cuh"
#include "gemm_tc.cuh"

namespace nmx {

constexpr int kLeafW = 32;      // recursion leaf width (the panel a leaf kernel factors)
constexpr int kLeafMax = 64;    // widest leaf the kernel supports
constexpr int kLeafThreads = 256;
constexpr int kTrsmLeaf = 32;

// One CTA's published pivot candidate for one column: |a|, its row, and the
// column number + 1 that marks the entry as current.
template <typename T>
struct LeafSlot {
    T mag;
    int row;
    int seq;
};

template <typename T>
struct LeafScratch {
    LeafSlot<T> *slots;  // [2][G]
    T *cand_rows;        // [2][G][kLeafMax] the candidate rows' panel values
    T *col_rows;         // [2][kLeafMax] row `col` as it was before the swap
    int *err;
};

__device__ __forceinline__ int ld_acquire_s32(const int *p) {
    int v;
    asm volatile("ld.acquire.gpu.global.s32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_release_s32(int *p, int v) {
    asm volatile("st.release.gpu.global.s32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

// Cooperative leaf: factor columns [c, c+w) (w <= kLeafMax) over rows [c, n)
// in place.  Each column is one exchange: every CTA publishes its candidate
// (value, row, the candidate row and, from its owner, row `col`) in its own
// slot with a sequence number, then waits until every slot carries the
// column's number -- the exchange is the barrier, no atomic counter.
template <typename T>
__global__ void __launch_bounds__(kLeafThreads)
    getrf_leaf_kernel(T *A, int64_t lda, int n, int c, int w, int rows_per_cta, int32_t *ipiv,
                      int32_t *info, LeafScratch<T> sc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ldl = w | 1;
    T *loc = reinterpret_cast<T *>(smem_raw);            // rows_per_cta x ldl
    T *prow = loc + (size_t)rows_per_cta * ldl;           // pivot row (w)
    __shared__ T s_mag[kLeafThreads / 32];
    __shared__ int s_row[kLeafThreads / 32];
    __shared__ int s_piv, s_wcta, s_fail;

    const int G = gridDim.x, cta = blockIdx.x, tid = threadIdx.x;
    const int lane = tid & 31, warp = tid >> 5;
    const int r0 = c + cta * rows_per_cta;                // first global row owned
    const int nloc = max(0, min(rows_per_cta, n - r0));   // rows owned

    for (int e = tid; e < nloc * w; e += kLeafThreads) {
        int r = e / w, j = e - r * w;
        loc[r * ldl + j] = A[(int64_t)(r0 + r) * lda + c + j];
    }
    if (tid == 0) s_fail = 0;
    __syncthreads();

    for (int j = 0; j < w; ++j) {
        const int col = c + j;
        const int slot = j & 1;
        // Local argmax over owned rows with global index >= col; zero and NaN
        // magnitudes never pivot (numax: strict > starting from 0).
        T best = T(-1);
        int brow = INT32_MAX;
        for (int r = tid; r < nloc; r += kLeafThreads) {
            const int gr = r0 + r;
            if (gr < col) continue;
            const T m = fabs(loc[r * ldl + j]);
            if (!(m > T(0))) continue;
            if (m > best || (m == best && gr < brow)) {
                best = m;
                brow = gr;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const T om = __shfl_xor_sync(0xffffffffu, best, o);
            const int orow = __shfl_xor_sync(0xffffffffu, brow, o);
            if (om > best || (om == best && orow < brow)) {
                best = om;
                brow = orow;
            }
        }
        if (lane == 0) {
            s_mag[warp] = best;
            s_row[warp] = brow;
        }
        __syncthreads();
        if (warp == 0) {
            best = lane < kLeafThreads / 32 ? s_mag[lane] : T(-1);
            brow = lane < kLeafThreads / 32 ? s_row[lane] : INT32_MAX;
            for (int o = 16; o > 0; o >>= 1) {
                const T om = __shfl_xor_sync(0xffffffffu, best, o);
                const int orow = __shfl_xor_sync(0xffffffffu, brow, o);
                if (om > best || (om == best && orow < brow)) {
                    best = om;
                    brow = orow;
                }
            }
            // Publish: the rows first, then the slot, then its sequence number.
            if (brow != INT32_MAX)
                for (int q = lane; q < w; q += 32)
                    sc.cand_rows[((size_t)slot * G + cta) * kLeafMax + q] =
                        loc[(brow - r0) * ldl + q];
            if (col >= r0 && col < r0 + nloc)
                for (int q = lane; q < w; q += 32)
                    sc.col_rows[slot * kLeafMax + q] = loc[(col - r0) * ldl + q];
            __threadfence();
            __syncwarp();
            if (lane == 0) {
                LeafSlot<T> *me = &sc.slots[slot * G + cta];
                me->mag = best;
                me->row = brow;
                __threadfence();
                st_release_s32(&me->seq, col + 1);
            }
            // Wait until every CTA's slot carries this column (bounded).
            long long spins = 0;
            bool ready = false;
            while (!ready) {
                bool mine = true;
                for (int g = lane; g < G; g += 32)
                    mine &= ld_acquire_s32(&sc.slots[slot * G + g].seq) == col + 1;
                ready = __all_sync(0xffffffffu, mine);
                if (!ready && ++spins > kSpinLimit) {
                    if (lane == 0) {
                        atomicExch(sc.err, 1);
                        s_fail = 1;
                    }
                    break;
                }
            }
            // Every CTA reduces the same candidates in the same order.
            if (ready) {
                best = T(-1);
                brow = INT32_MAX;
                int bcta = -1;
                for (int g = lane; g < G; g += 32) {
                    const T m = __ldcg(&sc.slots[slot * G + g].mag);
                    const int rr = __ldcg(&sc.slots[slot * G + g].row);
                    if (m > best || (m == best && rr < brow)) {
                        best = m;
                        brow = rr;
                        bcta = g;
                    }
                }
                for (int o = 16; o > 0; o >>= 1) {
                    const T om = __shfl_xor_sync(0xffffffffu, best, o);
                    const int orow = __shfl_xor_sync(0xffffffffu, brow, o);
                    const int octa = __shfl_xor_sync(0xffffffffu, bcta, o);
                    if (om > best || (om == best && orow < brow)) {
                        best = om;
                        brow = orow;
                        bcta = octa;
                    }
                }
                if (lane == 0) {
                    s_piv = brow;
                    s_wcta = bcta;
                }
            }
        }
        __syncthreads();
        if (s_fail) return;
        // No positive magnitude anywhere: numax keeps row `col` as the pivot.
        const bool none = s_piv == INT32_MAX;
        const int piv = none ? col : s_piv;
        // Published data is read through L2 (__ldcg): the same addresses held
        // the values of two columns ago.
        for (int q = tid; q < w; q += kLeafThreads)
            prow[q] = none ? __ldcg(&sc.col_rows[slot * kLeafMax + q])
                           : __ldcg(&sc.cand_rows[((size_t)slot * G + s_wcta) * kLeafMax + q]);
        __syncthreads();
        if (piv != col) {
            if (col >= r0 && col < r0 + nloc)
                for (int q = tid; q < w; q += kLeafThreads) loc[(col - r0) * ldl + q] = prow[q];
            if (piv >= r0 && piv < r0 + nloc)
                for (int q = tid; q < w; q += kLeafThreads)
                    loc[(piv - r0) * ldl + q] = __ldcg(&sc.col_rows[slot * kLeafMax + q]);
        }
        if (cta == 0 && tid == 0) {
            ipiv[col] = piv;
            if (none && *info == 0) *info = col + 1;
        }
        __syncthreads();
        T p = prow[j];
        if (p == T(0)) p = pivot_floor<T>::value;
        for (int r = tid; r < nloc; r += kLeafThreads) {
            const int gr = r0 + r;
            if (gr <= col) continue;
            const T l = loc[r * ldl + j] / p;
            loc[r * ldl + j] = l;
            for (int jj = j + 1; jj < w; ++jj) loc[r * ldl + jj] -= l * prow[jj];
        }
        __syncthreads();
    }
    for (int e = tid; e < nloc * w; e += kLeafThreads) {
        int r = e / w, j = e - r * w;
        A[(int64_t)(r0 + r) * lda + c + j] = loc[r * ldl + j];
    }
}

// Cluster leaf: the same panel factorization on one thread-block cluster
// (up to 16 CTAs, one per SM) whose shared memories together hold the whole
// panel.  The per-column exchange runs over distributed shared memory: each
// CTA leaves its candidate (|a|, row, the row's panel values) and, from the
// owner, row `col` in its own shared memory, one hardware cluster barrier,
// then every CTA reads the others' candidates and the winning row directly
// from their shared memory.  No global-memory round trip per column.
constexpr int kClusterLeafThreads = 512;

template <typename T>
__global__ void __launch_bounds__(kClusterLeafThreads)
    getrf_cluster_leaf_kernel(T *A, int64_t lda, int n, int c, int w, int rows_per_cta,
                              int32_t *ipiv, int32_t *info) {
    namespace cg = cooperative_groups;
    cg::cluster_group cluster = cg::this_cluster();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const int ldl = w | 1;
    T *loc = reinterpret_cast<T *>(smem_raw);                 // rows_per_cta x ldl
    T *xch = loc + (size_t)rows_per_cta * ldl;                 // [2][3][kLeafMax]
    // xch[slot][0] = candidate row, xch[slot][1] = row `col`, xch[slot][2] = pivot row
    __shared__ T s_cmag[2];
    __shared__ int s_crow[2];
    __shared__ T s_mag[kClusterLeafThreads / 32];
    __shared__ int s_row[kClusterLeafThreads / 32];
    __shared__ int s_piv, s_wcta;

    const int CS = (int)cluster.num_blocks(), cta = (int)cluster.block_rank();
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = kClusterLeafThreads / 32;
    const int r0 = c + cta * rows_per_cta;
    const int nloc = max(0, min(rows_per_cta, n - r0));
    const int col_owner = 0;  // row `col` is always within CTA (col - c) / rows_per_cta
    (void)col_owner;

    for (int e = tid; e < nloc * w; e += kClusterLeafThreads) {
        const int r = e / w, j = e - r * w;
        loc[r * ldl + j] = A[(int64_t)(r0 + r) * lda + c + j];
    }
    __syncthreads();

    for (int j = 0; j < w; ++j) {
        const int col = c + j;
        const int slot = j & 1;
        T *myx = xch + (size_t)slot * 3 * kLeafMax;
        T best = T(-1);
        int brow = INT32_MAX;
        for (int r = tid; r < nloc; r += kClusterLeafThreads) {
            const int gr = r0 + r;
            if (gr < col) continue;
            const T m = fabs(loc[r * ldl + j]);
            if (!(m > T(0))) continue;
            if (m > best || (m == best && gr < brow)) {
                best = m;
                brow = gr;
            }
        }
        for (int o = 16; o > 0; o >>= 1) {
            const T om = __shfl_xor_sync(0xffffffffu, best, o);
            const int orow = __shfl_xor_sync(0xffffffffu, brow, o);
            if (om > best || (om == best && orow < brow)) {
                best = om;
                brow = orow;
            }
        }
        if (lane == 0) {
            s_mag[warp] = best;
            s_row[warp] = brow;
        }
        __syncthreads();
        if (warp == 0) {
            best = lane < NW ? s_mag[lane] : T(-1);
            brow = lane < NW ? s_row[lane] : INT32_MAX;
            for (int o = 16; o > 0; o >>= 1) {
                const T om = __shfl_xor_sync(0xffffffffu, best, o);
                const int orow = __shfl_xor_sync(0xffffffffu, brow, o);
                if (om > best || (om == best && orow < brow)) {
                    best = om;
                    brow = orow;
                }
            }
            if (lane == 0) {
                s_cmag[slot] = best;
                s_crow[slot] = brow;
            }
            if (brow != INT32_MAX)
                for (int q = lane; q < w; q += 32) myx[q] = loc[(brow - r0) * ldl + q];
            if (col >= r0 && col < r0 + nloc)
                for (int q = lane; q < w; q += 32) myx[kLeafMax + q] = loc[(col - r0) * ldl + q];
        }
        cluster.sync();  // candidates and row `col` visible cluster-wide
        if (warp == 0) {
            best = T(-1);
            brow = INT32_MAX;
            int bcta = -1;
            if (lane < CS) {
                const T *rm = cluster.map_shared_rank(&s_cmag[slot], lane);
                const int *rr = cluster.map_shared_rank(&s_crow[slot], lane);
                best = *rm;
                brow = *rr;
                bcta = lane;
            }
            for (int o = 16; o > 0; o >>= 1) {
                const T om = __shfl_xor_sync(0xffffffffu, best, o);
                const int orow = __shfl_xor_sync(0xffffffffu, brow, o);
                const int octa = __shfl_xor_sync(0xffffffffu, bcta, o);
                if (om > best || (om == best && orow < brow)) {
                    best = om;
                    brow = orow;
                    bcta = octa;
                }
            }
            if (lane == 0) {
                s_piv = brow;
                s_wcta = bcta;
            }
        }
        __syncthreads();
        const bool none = s_piv == INT32_MAX;
        const int piv = none ? col : s_piv;
        const int col_cta = (col - c) / rows_per_cta;
        T *prow = myx + 2 * kLeafMax;
        if (tid < w) {
            const T *src = none ? cluster.map_shared_rank(xch + (size_t)slot * 3 * kLeafMax + kLeafMax,
                                                          col_cta)
                                : cluster.map_shared_rank(xch + (size_t)slot * 3 * kLeafMax, s_wcta);
            prow[tid] = src[tid];
        }
        __syncthreads();
        if (piv != col) {
            if (col >= r0 && col < r0 + nloc)
                for (int q = tid; q < w; q += kClusterLeafThreads) loc[(col - r0) * ldl + q] = prow[q];
            if (piv >= r0 && piv < r0 + nloc) {
                const T *oldcol =
                    cluster.map_shared_rank(xch + (size_t)slot * 3 * kLeafMax + kLeafMax, col_cta);
                for (int q = tid; q < w; q += kClusterLeafThreads)
                    loc[(piv - r0) * ldl + q] = oldcol[q];
            }
        }
        if (cta == 0 && tid == 0) {
            ipiv[col] = piv;
            if (none && *info == 0) *info = col + 1;
        }
        __syncthreads();
        T p = prow[j];
        if (p == T(0)) p = pivot_floor<T>::value;
        for (int r = tid; r < nloc; r += kClusterLeafThreads) {
            const int gr = r0 + r;
            if (gr <= col) continue;
            const T l = loc[r * ldl + j] / p;
            loc[r * ldl + j] = l;
            for (int jj = j + 1; jj < w; ++jj) loc[r * ldl + jj] -= l * prow[jj];
        }
        __syncthreads();
    }
    // No CTA may leave while others can still read its shared memory.
    cluster.sync();
    for (int e = tid; e < nloc * w; e += kClusterLeafThreads) {
        const int r = e / w, j = e - r * w;
        A[(int64_t)(r0 + r) * lda + c + j] = loc[r * ldl + j];
    }
}

// Apply interchanges ipiv[c..c+w) to the columns outside [c, c+w) of rows of
// A (ncols wide).  One thread per column, swaps in order.
template <typename T>
__global__ void laswp_kernel(T *A, int64_t lda, int ncols, int c, int w, const int32_t *ipiv,
                             int skip_lo, int skip_hi) {
    int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncols || (col >= skip_lo && col < skip_hi)) return;
    for (int s = 0; s < w; ++s) {
        int r1 = c + s, r2 = ipiv[c + s];
        if (r1 != r2) {
            T a = A[(int64_t)r1 * lda + col];
            A[(int64_t)r1 * lda + col] = A[(int64_t)r2 * lda + col];
            A[(int64_t)r2 * lda + col] = a;
        }
    }
}

// X := L^-1 X for the w x w (w <= 32) lower block L at (r, r) of A (unit or
// not) and X = rows [r, r+w) x cols [c0, c1) of B.  One thread per column.
// cp.async of one element (4 or 8 bytes) into shared memory.
template <typename T>
__device__ __forceinline__ void leaf_copy_async(T *dst, const T *src) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(d), "l"(src) : "memory");
}

template <typename T, bool UNIT>
__global__ void trsm_lower_leaf_kernel(const T *A, int64_t lda, int r, int w, T *B, int64_t ldb,
                                       int c0, int c1) {
    __shared__ T Ls[kTrsmLeaf][kTrsmLeaf + 1];
    // The block's copies all in flight (cp.async), then one wait.
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
        int i = e / w, j = e - i * w;
        leaf_copy_async(&Ls[i][j], &A[(int64_t)(r + i) * lda + r + j]);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    int col = c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= c1) return;
    T x[kTrsmLeaf];
#pragma unroll
    for (int i = 0; i < kTrsmLeaf; ++i) x[i] = i < w ? B[(int64_t)(r + i) * ldb + col] : T(0);
#pragma unroll
    for (int i = 0; i < kTrsmLeaf; ++i) {
        if (i < w) {
            T s = x[i];
#pragma unroll
            for (int p = 0; p < kTrsmLeaf; ++p)
                if (p < i) s -= Ls[i][p] * x[p];
            x[i] = UNIT ? s : s / Ls[i][i];
        }
    }
#pragma unroll
    for (int i = 0; i < kTrsmLeaf; ++i)
        if (i < w) B[(int64_t)(r + i) * ldb + col] = x[i];
}

// X := U^-1 X for the w x w upper block U at (r, r) of A (non-unit), or
// with TRANS the transpose of the lower block stored there (L^T).
template <typename T, bool TRANS>
__global__ void trsm_upper_leaf_kernel(const T *A, int64_t lda, int r, int w, T *B, int64_t ldb,
                                       int c0, int c1) {
    __shared__ T Us[kTrsmLeaf][kTrsmLeaf + 1];
    // The block's copies all in flight (cp.async; TRANS lands transposed).
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
        int i = e / w, j = e - i * w;
        leaf_copy_async(TRANS ? &Us[j][i] : &Us[i][j], &A[(int64_t)(r + i) * lda + r + j]);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    int col = c0 + blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= c1) return;
    T x[kTrsmLeaf];
#pragma unroll
    for (int i = 0; i < kTrsmLeaf; ++i) x[i] = i < w ? B[(int64_t)(r + i) * ldb + col] : T(0);
#pragma unroll
    for (int s = 0; s < kTrsmLeaf; ++s) {
        const int i = kTrsmLeaf - 1 - s;
        if (i < w) {
            T v = x[i];
#pragma unroll
            for (int p = 0; p < kTrsmLeaf; ++p)
                if (p > i && p < w) v -= Us[i][p] * x[p];
            x[i] = v / Us[i][i];
        }
    }
#pragma unroll
    for (int i = 0; i < kTrsmLeaf; ++i)
        if (i < w) B[(int64_t)(r + i) * ldb + col] = x[i];
}

// ---- host drivers -------------------------------------------------------

template <typename T>
struct LuRun {
    nmx_ctx ctx;
    cudaStream_t st;
    GemmSub gs;
    T *A;
    int64_t lda;
    int n;
    int32_t *ipiv;
    int32_t *info;
    LeafScratch<T> sc;
    int max_ctas;
    int cluster;  // CTAs per cluster for the cluster leaf (0: not available)
    int max_w;    // widest leaf (multiple of 8, <= kLeafMax)
    bool tournament = false;  // tournament-pivoting leaves (FP32 only)
    CaluScratch cs = {};
    // Tournament leaves: the columns their row interchanges reach now (the
    // look-ahead panel; [0, n) unblocked) and where they leave their row
    // moves for the other columns.
    int scope_lo = 0, scope_hi = 0;
    int *lists = nullptr;
    int nlists = 0;
    bool keep_lists = false;  // the lists are applied later (look-ahead panel)
};

// Shared-memory bytes the cluster leaf needs for an m-row panel of width w.
template <typename T>
static size_t cluster_leaf_smem(int m, int w, int cs) {
    const size_t rpc = (size_t)ceil_div(m, cs);
    return sizeof(T) * (rpc * (size_t)(w | 1) + 6 * (size_t)kLeafMax);
}

// Widest leaf (multiple of 8, <= R.max_w) the cluster leaf can hold for an
// m-row panel; R.max_w if even 8 columns do not fit (the cooperative leaf
// runs).
template <typename T>
static int leaf_width(const LuRun<T> &R, int m) {
    if (R.tournament) return std::min(R.max_w, kCaluW);
    if (R.cluster <= 0) return R.max_w;
    for (int w = R.max_w; w >= 8; w -= 8)
        if (cluster_leaf_smem<T>(m, w, R.cluster) + 2048 <= R.ctx->smem_optin) return w;
    return R.max_w;
}

// Row moves of `nlists` leaves in columns [a0, a1) and [b0, b1).
template <typename T>
static int calu_swap(cudaStream_t st, T *A, int64_t lda, const int *lists, int nlists, int a0,
                     int a1, int b0, int b1) {
    const int cols = std::max(0, a1 - a0) + std::max(0, b1 - b0);
    if (cols == 0 || nlists == 0) return 0;
    calu_swap_kernel<T><<<(unsigned)ceil_div(cols, kCaluApplyThreads), kCaluApplyThreads, 0, st>>>(
        A, lda, lists, nlists, a0, std::max(a0, a1), b0, std::max(b0, b1));
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

// The next slot for a leaf's row moves.  Unblocked the slots recycle (each
// list is applied at once); a look-ahead panel keeps all of its leaves'
// lists, and the panel widths are chosen so they fit -- nullptr otherwise.
template <typename T>
static int *leaf_list(LuRun<T> &R) {
    if (R.nlists >= kCaluMaxLists) {
        if (R.keep_lists) {
            set_error("LU panel needs more than %d leaf move lists", kCaluMaxLists);
            return nullptr;
        }
        R.nlists = 0;
    }
    return R.lists + (size_t)R.nlists++ * kCaluListStride;
}

// A partial-pivoting leaf's interchanges on the other columns in scope: as a
// row-move list for leaves of <= 32 columns, else swap by swap (unblocked
// runs only).
template <typename T>
static int leaf_swap(LuRun<T> &R, int c, int w) {
    if (w <= kCaluW) {
        int *ml = leaf_list(R);
        if (!ml) return NMX_ERR_INTERNAL;
        ipiv_moves_kernel<<<1, 32, 0, R.st>>>(R.ipiv, c, w, ml);
        NMX_CUDA_TRY(cudaGetLastError());
        return calu_swap<T>(R.st, R.A, R.lda, ml, 1, R.scope_lo, c, c + w, R.scope_hi);
    }
    const int threads = 256;
    laswp_kernel<T><<<(unsigned)ceil_div(R.n, threads), threads, 0, R.st>>>(R.A, R.lda, R.n, c, w,
                                                                             R.ipiv, c, c + w);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

// Tournament-pivoting leaf: the pivot search, the panel's rows into place,
// and the row moves across the columns in scope.
static int calu_leaf(LuRun<float> &R, int c, int w) {
    const int m = R.n - c;
    const int nctas = (int)ceil_div(m, kCaluRows);
    const bool vec = R.lda % 4 == 0 && reinterpret_cast<uintptr_t>(R.A) % 16 == 0;
    int *ml = leaf_list(R);
    if (!ml) return NMX_ERR_INTERNAL;
    calu_pick_kernel<<<nctas, kCaluThreads, 0, R.st>>>(R.A, R.lda, R.n, c, w, nctas, vec, R.cs,
                                                    R.ipiv, R.info, ml);
    // The panel's rows and, in the same launch, the moves in the other
    // columns in scope.
    const int panel = (int)ceil_div(m, kCaluApplyThreads);
    const int cols = (c - R.scope_lo) + (R.scope_hi - c - w);
    calu_apply_kernel<<<(unsigned)(panel + ceil_div(cols, kCaluApplyThreads)), kCaluApplyThreads,
                        kCaluApplySmem, R.st>>>(R.A, R.lda, R.n, c, w, R.cs, ml, panel,
                                                R.scope_lo, c, c + w, R.scope_hi);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

template <typename T>
static int leaf(LuRun<T> &R, int c, int w) {
    const int m = R.n - c;
    if constexpr (std::is_same<T, float>::value) {
        if (R.tournament) return calu_leaf(R, c, w);
    }
    if (R.cluster > 0 && cluster_leaf_smem<T>(m, w, R.cluster) + 2048 <= R.ctx->smem_optin) {
        int rpc = (int)ceil_div(m, R.cluster);
        cudaLaunchConfig_t cfg = {};
        cfg.gridDim = dim3(R.cluster);
        cfg.blockDim = dim3(kClusterLeafThreads);
        cfg.dynamicSmemBytes = cluster_leaf_smem<T>(m, w, R.cluster);
        cfg.stream = R.st;
        cudaLaunchAttribute attr[1];
        attr[0].id = cudaLaunchAttributeClusterDimension;
        attr[0].val.clusterDim.x = R.cluster;
        attr[0].val.clusterDim.y = 1;
        attr[0].val.clusterDim.z = 1;
        cfg.attrs = attr;
        cfg.numAttrs = 1;
        NMX_CUDA_TRY(cudaLaunchKernelEx(&cfg, getrf_cluster_leaf_kernel<T>, R.A, R.lda, R.n, c, w,
                                        rpc, R.ipiv, R.info));
        return leaf_swap(R, c, w);
    }
    int G = (int)std::min<int64_t>(R.max_ctas, ceil_div(m, 32));
    G = std::max(G, 1);
    int rpc = (int)ceil_div(m, G);
    G = (int)ceil_div(m, rpc);
    size_t smem = sizeof(T) * ((size_t)rpc * (w | 1) + kLeafMax);
    if (smem > R.ctx->smem_optin - 1024) {
        set_error("matrix order %d too large for the leaf panel (%zu B shared)", R.n, smem);
        return NMX_ERR_UNSUPPORTED;
    }
    void *args[] = {&R.A, &R.lda, &R.n, &c, &w, &rpc, &R.ipiv, &R.info, &R.sc};
    NMX_CUDA_TRY(cudaLaunchCooperativeKernel((void *)getrf_leaf_kernel<T>, dim3(G),
                                             dim3(kLeafThreads), args, smem, R.st));
    return leaf_swap(R, c, w);
}

// X := L^-1 X, L the w x w lower block at (r, r) of A, X rows [r, r+w) cols [c0, c1) of B.
template <typename T, bool UNIT>
int trsm_lower(const GemmSub &gs, const T *A, int64_t lda, int r, int w, T *B, int64_t ldb, int c0,
               int c1) {
    cudaStream_t st = gs.st;
    if (w <= 0 || c1 <= c0) return 0;
    if constexpr (UNIT && sizeof(T) == 8) {
        // Unit lower blocks of 64..256 rows (multiples of 32): one kernel.
        if (w > kTrsmLeaf && w <= kTrsmMaxW && w % 32 == 0) {
            static bool attr_set[64] = {};
            int dev = 0;
            NMX_CUDA_TRY(cudaGetDevice(&dev));
            if (dev < 64 && !attr_set[dev]) {
                NMX_CUDA_TRY(cudaFuncSetAttribute(trsm_unit_lower_t_kernel<T>,
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)trsm_unit_lower_t_smem<T>(kTrsmMaxW)));
                attr_set[dev] = true;
            }
            trsm_unit_lower_t_kernel<T><<<(unsigned)ceil_div(c1 - c0, 32), kTrsmThreads,
                                          trsm_unit_lower_t_smem<T>(w), st>>>(A, lda, r, w, B, ldb,
                                                                              c0, c1);
            NMX_CUDA_TRY(cudaGetLastError());
            return 0;
        }
    }
    if (w <= kTrsmLeaf) {
        int threads = 128;
        trsm_lower_leaf_kernel<T, UNIT>
            <<<(unsigned)ceil_div(c1 - c0, threads), threads, 0, st>>>(A, lda, r, w, B, ldb, c0, c1);
        NMX_CUDA_TRY(cudaGetLastError());
        return 0;
    }
    int hw = (w / 2 + kTrsmLeaf - 1) / kTrsmLeaf * kTrsmLeaf;
    int rc = trsm_lower<T, UNIT>(gs, A, lda, r, hw, B, ldb, c0, c1);
    if (rc) return rc;
    rc = gs(w - hw, c1 - c0, hw, A + (int64_t)(r + hw) * lda + r, lda, B + (int64_t)r * ldb + c0, ldb,
            B + (int64_t)(r + hw) * ldb + c0, ldb);
    if (rc) return rc;
    return trsm_lower<T, UNIT>(gs, A, lda, r + hw, w - hw, B, ldb, c0, c1);
}

// X := U^-1 X (TRANS: X := L^-T X with L the lower block stored at (r, r)).
template <typename T, bool TRANS>
int trsm_upper(const GemmSub &gs, const T *A, int64_t lda, int r, int w, T *B, int64_t ldb, int c0,
               int c1) {
    cudaStream_t st = gs.st;
    if (w <= 0 || c1 <= c0) return 0;
    if (w <= kTrsmLeaf) {
        int threads = 128;
        trsm_upper_leaf_kernel<T, TRANS>
            <<<(unsigned)ceil_div(c1 - c0, threads), threads, 0, st>>>(A, lda, r, w, B, ldb, c0, c1);
        NMX_CUDA_TRY(cudaGetLastError());
        return 0;
    }
    int hw = (w / 2 + kTrsmLeaf - 1) / kTrsmLeaf * kTrsmLeaf;
    int rc = trsm_upper<T, TRANS>(gs, A, lda, r + hw, w - hw, B, ldb, c0, c1);
    if (rc) return rc;
    // B_top -= U_top,bot X_bot   (TRANS: U_top,bot = (L_bot,top)^T, the
    // (w - hw) x hw block below the diagonal read transposed).
    if (TRANS) {
        rc = gemm_cc<T>(st, true, false, hw, c1 - c0, w - hw, T(-1),
                        A + (int64_t)(r + hw) * lda + r, lda, B + (int64_t)(r + hw) * ldb + c0, ldb,
                        T(1), B + (int64_t)r * ldb + c0, ldb);
        if (rc) return rc;
    } else {
        rc = gs(hw, c1 - c0, w - hw, A + (int64_t)r * lda + r + hw, lda,
                B + (int64_t)(r + hw) * ldb + c0, ldb, B + (int64_t)r * ldb + c0, ldb);
        if (rc) return rc;
    }
    return trsm_upper<T, TRANS>(gs, A, lda, r, hw, B, ldb, c0, c1);
}

// X := L^-1 X (unit lower L, w x w at (r, r) of A; X rows [r, r+w) x cols
// [c0, c1) of B) for the tournament LU: one kernel for w <= 256 in multiples
// of 32, else the recursion.
static int trsm_unit_lower_f32(const GemmSub &gs, const float *A, int64_t lda, int r, int w,
                               float *B, int64_t ldb, int c0, int c1) {
    if (w <= 0 || c1 <= c0) return 0;
    if (w > kTrsmMaxW || w % 32 != 0) return trsm_lower<float, true>(gs, A, lda, r, w, B, ldb, c0, c1);
    static bool attr_set[64] = {};
    int dev = 0;
    NMX_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 64 && !attr_set[dev]) {
        NMX_CUDA_TRY(cudaFuncSetAttribute(trsm_unit_lower_kernel,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)trsm_unit_lower_smem(kTrsmMaxW)));
        attr_set[dev] = true;
    }
    trsm_unit_lower_kernel<<<(unsigned)ceil_div(c1 - c0, 32), kTrsmThreads, trsm_unit_lower_smem(w),
                             gs.st>>>(A, lda, r, w, B, ldb, c0, c1);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

template <typename T>
static int getrf2(LuRun<T> &R, int c, int w) {
    const int lw = leaf_width<T>(R, R.n - c);
    if (w <= lw) return leaf<T>(R, c, w);
    // Split on multiples of the leaf width (a multiple of 8, which keeps every
    // block offset 16-byte aligned for the tensor-core update).
    int hw = std::min(w - 1, (w / 2 + lw - 1) / lw * lw);
    int rc = getrf2<T>(R, c, hw);
    if (rc) return rc;
    // U12 := L11^-1 A12 over the right half's columns.
    if constexpr (std::is_same<T, float>::value) {
        if (R.tournament)
            rc = trsm_unit_lower_f32(R.gs, R.A, R.lda, c, hw, R.A, R.lda, c + hw, c + w);
        else
            rc = trsm_lower<T, true>(R.gs, R.A, R.lda, c, hw, R.A, R.lda, c + hw, c + w);
    } else {
        rc = trsm_lower<T, true>(R.gs, R.A, R.lda, c, hw, R.A, R.lda, c + hw, c + w);
    }
    if (rc) return rc;
    // A22 -= L21 U12.
    rc = R.gs(R.n - c - hw, w - hw, hw, R.A + (int64_t)(c + hw) * R.lda + c, R.lda,
              R.A + (int64_t)c * R.lda + c + hw, R.lda, R.A + (int64_t)(c + hw) * R.lda + c + hw,
              R.lda);
    if (rc) return rc;
    return getrf2<T>(R, c + hw, w - hw);
}

// Right-looking LU over panels of nb columns with a look-ahead of one panel
// (tournament leaves only).  Two streams: the panel stream (high priority)
// updates the next panel's columns and factors it while the update stream
// applies the previous panel to every other column:
//
//   panel stream, step i:  moves(i) + U12 + GEMM on panel i+1's columns,
//                          then factor panel i+1 (its leaves' row moves
//                          reach panel i+1's columns only, the rest is kept);
//   update stream, step i: moves(i) on columns [0, i nb) and past panel
//                          i+1, U12 and the GEMM past panel i+1.
//
// Step i's two halves touch disjoint columns and only read panel i.  The
// panel stream starts step i+1 after the update stream's step i (which
// updated panel i+2's columns); the update stream starts step i after panel
// i is factored.  The leaves' move lists alternate between two buffers.
// U12 := L11^-1 A12 for the look-ahead steps.
template <typename T>
static int la_trsm(const GemmSub &gs, bool tournament, T *A, int64_t lda, int k, int kb, int c0,
                   int c1) {
    if constexpr (std::is_same<T, float>::value) {
        if (tournament) return trsm_unit_lower_f32(gs, A, lda, k, kb, A, lda, c0, c1);
    }
    return trsm_lower<T, true>(gs, A, lda, k, kb, A, lda, c0, c1);
}

template <typename T>
static int getrf_lookahead(LuRun<T> &R, int nb) {
    nmx_ctx ctx = R.ctx;
    const int n = R.n;
    int rc = ctx_lookahead_streams(ctx);
    if (rc) return rc;
    cudaStream_t P = ctx->la_stream[0], U = ctx->la_stream[1];
    cudaEvent_t eP = ctx->la_event[0], eU = ctx->la_event[1];
    GemmSub gP = R.gs, gU = R.gs;
    gP.st = P;
    gU.st = U;
    // Optionally the update stream's tensor-core GEMMs leave SMs to the panel
    // stream (a static persistent GEMM on the rest).  Off by default: the
    // hardware-scheduled GEMM already interleaves the panel's kernels.
    const int64_t keep = ctx->tune_lu_panel_sms < 0 ? 0 : ctx->tune_lu_panel_sms;
    gU.sm_limit = keep > 0 ? (int)std::max<int64_t>(16, ctx->sm_count - keep) : 0;
    if (gP.precision) {
        gP.ws_bytes = tc_gemm_workspace_bytes(n, nb, nb, gP.precision) + 4096;
        rc = ctx->ensure_slot(kWsGemm16Panel, gP.ws_bytes, &gP.ws);
        if (rc) return rc;
    }
    LuRun<T> RP = R;
    RP.st = P;
    RP.gs = gP;
    RP.keep_lists = true;
    int *buf[2] = {R.cs.lists, R.cs.lists + (size_t)kCaluMaxLists * kCaluListStride};
    int cur = 0;
    auto panel = [&](int k, int kb) {
        RP.scope_lo = k;
        RP.scope_hi = k + kb;
        RP.lists = buf[cur];
        RP.nlists = 0;
        return getrf2<T>(RP, k, kb);
    };
    auto body = [&]() -> int {
        NMX_CUDA_TRY(cudaEventRecord(eU, R.st));
        NMX_CUDA_TRY(cudaStreamWaitEvent(P, eU, 0));
        NMX_CUDA_TRY(cudaStreamWaitEvent(U, eU, 0));
        int k = 0, kb = std::min(nb, n);
        int r = panel(k, kb);
        if (r) return r;
        NMX_CUDA_TRY(cudaEventRecord(eP, P));
        T *A = R.A;
        const int64_t lda = R.lda;
        while (k + kb < n) {
            const int next = k + kb, kb2 = std::min(nb, n - next), rest = next + kb2;
            const int *lst = buf[cur];
            const int nl = RP.nlists;
            NMX_CUDA_TRY(cudaStreamWaitEvent(U, eP, 0));
            NMX_CUDA_TRY(cudaStreamWaitEvent(P, eU, 0));
            // Panel stream: the next panel's columns, then the next panel.
            r = calu_swap<T>(P, A, lda, lst, nl, next, rest, 0, 0);
            if (r) return r;
            r = la_trsm<T>(gP, R.tournament, A, lda, k, kb, next, rest);
            if (r) return r;
            r = gP(n - next, kb2, kb, A + (int64_t)next * lda + k, lda, A + (int64_t)k * lda + next,
                   lda, A + (int64_t)next * lda + next, lda);
            if (r) return r;
            cur ^= 1;
            r = panel(next, kb2);
            if (r) return r;
            NMX_CUDA_TRY(cudaEventRecord(eP, P));
            // Update stream: everything else.
            r = calu_swap<T>(U, A, lda, lst, nl, 0, k, rest, n);
            if (r) return r;
            if (rest < n) {
                r = la_trsm<T>(gU, R.tournament, A, lda, k, kb, rest, n);
                if (r) return r;
                r = gU(n - next, n - rest, kb, A + (int64_t)next * lda + k, lda,
                       A + (int64_t)k * lda + rest, lda, A + (int64_t)next * lda + rest, lda);
                if (r) return r;
            }
            NMX_CUDA_TRY(cudaEventRecord(eU, U));
            k = next;
            kb = kb2;
        }
        // The last panel's moves on the columns before it.
        NMX_CUDA_TRY(cudaStreamWaitEvent(U, eP, 0));
        r = calu_swap<T>(U, A, lda, buf[cur], RP.nlists, 0, k, 0, 0);
        if (r) return r;
        NMX_CUDA_TRY(cudaEventRecord(eU, U));
        NMX_CUDA_TRY(cudaStreamWaitEvent(R.st, eU, 0));
        return 0;
    };
    rc = body();
    if (rc) {
        // On an error the caller's stream still waits for whatever both
        // streams already hold, so nothing queued there outlives the call's
        // ordering.
        cudaEventRecord(eP, P);
        cudaStreamWaitEvent(R.st, eP, 0);
        cudaEventRecord(eU, U);
        cudaStreamWaitEvent(R.st, eU, 0);
    }
    return rc;
}

int64_t tournament_max_rows() { return (int64_t)kCaluMaxCtas * kCaluRows; }

template <typename T>
void laswp_rows(cudaStream_t st, T *B, int64_t ldb, int n, int ncols, const int32_t *ipiv) {
    const int threads = 128;
    laswp_kernel<T><<<(unsigned)ceil_div(ncols, threads), threads, 0, st>>>(B, ldb, ncols, 0, n,
                                                                          ipiv, 0, 0);
}
template void laswp_rows<double>(cudaStream_t, double *, int64_t, int, int, const int32_t *);
template void laswp_rows<float>(cudaStream_t, float *, int64_t, int, int, const int32_t *);

template <typename T>
int getrf_run(nmx_ctx ctx, const GemmSub &gs, int64_t n, T *A, int64_t lda, int32_t *ipiv,
              int32_t *info, bool tournament) {
    cudaStream_t st = gs.st;
    NMX_CUDA_TRY(cudaMemsetAsync(info, 0, sizeof(int32_t), st));
    if (n == 0) return 0;
    const int G = ctx->sm_count;
    const size_t slot_bytes = sizeof(LeafSlot<T>) * 2 * (size_t)G;
    size_t bytes = slot_bytes + sizeof(T) * (2 * (size_t)G * kLeafMax + 2 * kLeafMax) + 64;
    void *wsv = nullptr;
    int rc = ctx->ensure_slot(kWsLeaf, bytes, &wsv);
    if (rc) return rc;
    char *ws = static_cast<char *>(wsv);
    LeafScratch<T> sc;
    sc.slots = reinterpret_cast<LeafSlot<T> *>(ws);
    sc.cand_rows = reinterpret_cast<T *>(ws + slot_bytes);
    sc.col_rows = sc.cand_rows + 2 * (size_t)G * kLeafMax;
    sc.err = reinterpret_cast<int *>(sc.col_rows + 2 * kLeafMax);
    // Sequence numbers start below every column's (col + 1 >= 1).
    NMX_CUDA_TRY(cudaMemsetAsync(sc.slots, 0, slot_bytes, st));
    NMX_CUDA_TRY(cudaMemsetAsync(sc.err, 0, sizeof(int), st));
    const int leaf_ctas = ctx->tune_lu_leaf_ctas > 0
                              ? (int)std::min<int64_t>(ctx->tune_lu_leaf_ctas, G)
                              : G;
    // Every CTA of the cooperative leaf must be resident at once.
    int per_sm = 0;
    const int m = (int)n;
    int rpc_max = (int)ceil_div(m, std::min<int64_t>(leaf_ctas, ceil_div(m, 32)));
    size_t smem = sizeof(T) * ((size_t)rpc_max * (kLeafW | 1) + kLeafMax);
    NMX_CUDA_TRY(cudaFuncSetAttribute(getrf_leaf_kernel<T>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)std::min<size_t>(smem, ctx->smem_optin - 1024)));
    NMX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, getrf_leaf_kernel<T>,
                                                               kLeafThreads, smem));
    if (per_sm < 1) {
        set_error("matrix order %lld too large for the leaf panel", (long long)n);
        return NMX_ERR_UNSUPPORTED;
    }
    // Thread-block cluster for the cluster leaf: 16 CTAs (non-portable) when
    // the device can co-schedule them, else 8, else none.
    int cluster = 0;
    {
        auto kern = getrf_cluster_leaf_kernel<T>;
        const size_t smax = ctx->smem_optin - 2048;
        if (cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smax) ==
            cudaSuccess) {
            for (int cs : {16, 8}) {
                if (cs > 8 &&
                    cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) !=
                        cudaSuccess) {
                    cudaGetLastError();
                    continue;
                }
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3(cs);
                cfg.blockDim = dim3(kClusterLeafThreads);
                cfg.dynamicSmemBytes = smax;
                cudaLaunchAttribute attr[1];
                attr[0].id = cudaLaunchAttributeClusterDimension;
                attr[0].val.clusterDim.x = cs;
                attr[0].val.clusterDim.y = 1;
                attr[0].val.clusterDim.z = 1;
                cfg.attrs = attr;
                cfg.numAttrs = 1;
                int clusters = 0;
                if (cudaOccupancyMaxActiveClusters(&clusters, kern, &cfg) == cudaSuccess &&
                    clusters >= 1) {
                    cluster = cs;
                    break;
                }
                cudaGetLastError();
            }
        } else {
            cudaGetLastError();
        }
    }
    // A tuned cluster size is rounded down to a power of two no larger than
    // the one the device can co-schedule; 0 selects the cooperative leaf.
    if (ctx->tune_lu_cluster >= 0) {
        int cs = 0;
        for (int p = 16; p >= 1; p /= 2)
            if (p <= cluster && p <= ctx->tune_lu_cluster) {
                cs = p;
                break;
            }
        cluster = cs;
    }
    const int max_w = ctx->tune_lu_leaf_w > 0
                          ? (int)std::min<int64_t>(kLeafMax, ctx->tune_lu_leaf_w / 8 * 8)
                          : kLeafW;
    LuRun<T> R{ctx, st, gs, A, lda, (int)n, ipiv, info, sc, leaf_ctas, cluster, std::max(8, max_w)};
    // Every leaf leaves its row moves in a list (applied at once, or later to
    // the columns outside a look-ahead panel).
    void *cv = nullptr;
    rc = ctx->ensure_slot(kWsCalu, CaluScratch::bytes(), &cv);
    if (rc) return rc;
    R.cs.carve(cv);
    R.scope_lo = 0;
    R.scope_hi = (int)n;
    R.lists = R.cs.lists;
    // Tournament pivoting: FP32 panels of up to 131072 rows.
    if (std::is_same<T, float>::value && tournament && n <= (int64_t)kCaluMaxCtas * kCaluRows) {
        NMX_CUDA_TRY(cudaMemsetAsync(R.cs.count, 0, sizeof(unsigned) * (kCaluGroup + 1), st));
        R.tournament = true;
    }
    // Look-ahead panel width: a multiple of 32 in [64, 1024] (tournament
    // leaves), [64, 512] otherwise (leaves as narrow as 8 columns must fit
    // the panel's move lists); leaves of more than 32 columns run unblocked.
    // With numax's pivots the look-ahead starts at order 4096 by default (a
    // tuned width applies from two panels): below that the leaves' latency
    // is all there is to hide, and the unblocked recursion keeps its
    // summation order.
    {
        const bool tuned = ctx->tune_lu_lookahead >= 0;
        const int64_t want = tuned ? ctx->tune_lu_lookahead : 256;
        const int nb = (int)std::min<int64_t>(R.tournament ? 1024 : 512, want / 32 * 32);
        const int64_t from = (R.tournament || tuned) ? 2 * nb : std::max(2 * nb, 4096);
        // With numax's pivots every leaf must be a cluster leaf: a cooperative
        // grid leaf on the panel stream could not count on all its CTAs being
        // resident beside the update stream's kernels.
        const bool leaves_ok =
            R.tournament ||
            (R.cluster > 0 && cluster_leaf_smem<T>((int)n, 8, R.cluster) + 2048 <= ctx->smem_optin);
        if (nb >= 64 && n >= from && R.max_w <= kCaluW && leaves_ok)
            return getrf_lookahead(R, nb);
    }
    return getrf2<T>(R, 0, (int)n);
}

template int getrf_run<double>(nmx_ctx, const GemmSub &, int64_t, double *, int64_t, int32_t *,
                               int32_t *, bool);
template int getrf_run<float>(nmx_ctx, const GemmSub &, int64_t, float *, int64_t, int32_t *,
                              int32_t *, bool);

template <typename T>
static int getrf(nmx_ctx ctx, int64_t n, T *A, int64_t lda, int32_t *ipiv, int32_t *info,
                 void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(n >= 0 && n <= (1 << 20), 2, "n out of range");
    NMX_ARG_CHECK(A != nullptr || n == 0, 3, "A is NULL");
    NMX_ARG_CHECK(lda >= std::max<int64_t>(1, n), 4, "lda < max(1, n)");
    NMX_ARG_CHECK(ipiv != nullptr || n == 0, 5, "ipiv is NULL");
    NMX_ARG_CHECK(info != nullptr, 6, "info is NULL");
    DeviceGuard g(ctx->device);
    GemmSub gs;
    gs.st = static_cast<cudaStream_t>(stream);
    return getrf_run<T>(ctx, gs, n, A, lda, ipiv, info, ctx->tune_lu_tournament == 1);
}

template <typename T>
static int getrs(nmx_ctx ctx, int64_t n, int64_t nrhs, const T *LU, int64_t lda,
                 const int32_t *ipiv, T *B, int64_t ldb, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(n >= 0, 2, "n < 0");
    NMX_ARG_CHECK(nrhs >= 0, 3, "nrhs < 0");
    NMX_ARG_CHECK(LU != nullptr || n == 0, 4, "LU is NULL");
    NMX_ARG_CHECK(lda >= std::max<int64_t>(1, n), 5, "lda < max(1, n)");
    NMX_ARG_CHECK(ipiv != nullptr || n == 0, 6, "ipiv is NULL");
    NMX_ARG_CHECK(B != nullptr || n == 0 || nrhs == 0, 7, "B is NULL");
    NMX_ARG_CHECK(ldb >= std::max<int64_t>(1, nrhs), 8, "ldb < max(1, nrhs)");
    if (n == 0 || nrhs == 0) return 0;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    GemmSub gs;
    gs.st = st;
    int rc = 0;
    int threads = 128;
    laswp_kernel<T><<<(unsigned)ceil_div(nrhs, threads), threads, 0, st>>>(B, ldb, (int)nrhs, 0,
                                                                           (int)n, ipiv, 0, 0);
    NMX_CUDA_TRY(cudaGetLastError());
    rc = trsm_lower<T, true>(gs, LU, lda, 0, (int)n, B, ldb, 0, (int)nrhs);
    if (rc) return rc;
    return trsm_upper<T, false>(gs, LU, lda, 0, (int)n, B, ldb, 0, (int)nrhs);
}

// Explicit instantiations used by the Cholesky and IR drivers.
template int trsm_lower<double, true>(const GemmSub &, const double *, int64_t, int, int, double *,
                                    int64_t, int, int);
template int trsm_lower<float, true>(const GemmSub &, const float *, int64_t, int, int, float *,
                                    int64_t, int, int);
template int trsm_lower<double, false>(const GemmSub &, const double *, int64_t, int, int, double *,
                                    int64_t, int, int);
template int trsm_lower<float, false>(const GemmSub &, const float *, int64_t, int, int, float *,
                                    int64_t, int, int);
template int trsm_upper<double, true>(const GemmSub &, const double *, int64_t, int, int, double *,
                                    int64_t, int, int);
template int trsm_upper<float, true>(const GemmSub &, const float *, int64_t, int, int, float *,
                                    int64_t, int, int);
template int trsm_upper<double, false>(const GemmSub &, const double *, int64_t, int, int, double *,
                                    int64_t, int, int);
template int trsm_upper<float, false>(const GemmSub &, const float *, int64_t, int, int, float *,
                                    int64_t, int, int);

}  // namespace nmx

extern "C" {

NMX_API int nmx_getrf_f64(nmx_ctx ctx, int64_t n, double *A, int64_t lda, int32_t *ipiv,
                          int32_t *info, void *stream) {
    return nmx::getrf<double>(ctx, n, A, lda, ipiv, info, stream);
}
NMX_API int nmx_getrf_f32(nmx_ctx ctx, int64_t n, float *A, int64_t lda, int32_t *ipiv,
                          int32_t *info, void *stream) {
    return nmx::getrf<float>(ctx, n, A, lda, ipiv, info, stream);
}
NMX_API int nmx_getrs_f64(nmx_ctx ctx, int64_t n, int64_t nrhs, const double *LU, int64_t lda,
                          const int32_t *ipiv, double *B, int64_t ldb, void *stream) {
    return nmx::getrs<double>(ctx, n, nrhs, LU, lda, ipiv, B, ldb, stream);
}
NMX_API int nmx_getrs_f32(nmx_ctx ctx, int64_t n, int64_t nrhs, const float *LU, int64_t lda,
                          const int32_t *ipiv, float *B, int64_t ldb, void *stream) {
    return nmx::getrs<float>(ctx, n, nrhs, LU, lda, ipiv, B, ldb, stream);
}

}  // extern "C"
