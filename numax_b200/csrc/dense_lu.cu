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

#include "dense_common.cuh"

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

// ---- tournament-pivoting leaf (FP32: the mixed-precision factorization) ----
//
// The FP32 factorization inside iterative refinement (ir.cu) needs a stable
// LU, not numax's exact pivot sequence: refinement in FP64 makes the solution
// independent of which stable pivots the factors used.  Its leaves use
// tournament pivoting (CALU; Grigori, Demmel & Xiang, SIAM J. Matrix Anal.
// Appl. 32(4), 2011) over a reduction tree of at most three levels:
//   1. every CTA holds 512 rows of the panel, one row per thread in
//      registers, runs partial pivoting on them and publishes the (up to) w
//      rows it picked;
//   2. the last CTA of each group of 16 to finish (an arrival counter; no CTA
//      waits for another) stacks the group's 16 x w candidates -- their
//      original values, re-read from A -- and keeps the w rows partial
//      pivoting picks among them;
//   3. the last group to finish does the same over the groups' candidates,
//      keeping the multipliers: the rows it picks, in pick order, are the
//      pivot rows and hold L11\U11.  It writes them, the LAPACK-style
//      interchanges and the list of rows that change place.
// A second kernel solves every other row against U11 (l = a U11^-1, rows
// independent) and moves rows to their final positions across the whole
// width.  The pivot search costs one CTA barrier per column instead of one
// grid- or cluster-wide exchange.  A zero U11 diagonal is floored to 1e-30
// and the first one reported in info; a column without a nonzero candidate
// picks the lowest row.
constexpr int kCaluRows = 512;                          // rows per CTA, one per thread
constexpr int kCaluW = 32;                              // widest leaf
constexpr int kCaluWarps = kCaluRows / 32;
constexpr int kCaluGroup = kCaluRows / kCaluW;          // candidate sets one CTA stacks
constexpr int kCaluMaxCtas = kCaluGroup * kCaluGroup;   // panels of up to 131072 rows
constexpr int kCaluApplyThreads = 256;

struct CaluScratch {
    int *cand;        // [kCaluMaxCtas][kCaluW] first-level picks (global rows, -1: none)
    int *gcand;       // [kCaluGroup][kCaluW] second-level picks
    unsigned *count;  // [kCaluGroup + 1] arrival counters, zero between leaves
    float *lu;        // [kCaluW][kCaluW] L11\U11 of the pivot rows, pivot order
    int *gp;          // [kCaluW] pivot rows in pivot order (-1 past the panel)
    int *moves;       // [2 kCaluW][2] (from, to) of every row that changes place
    int *nmoves;      // 1
    static size_t bytes() {
        return sizeof(int) * ((size_t)kCaluMaxCtas * kCaluW + kCaluGroup * kCaluW + kCaluGroup +
                              1 + kCaluW + 4 * kCaluW + 1) +
               sizeof(float) * kCaluW * kCaluW + 256;
    }
    void carve(void *base) {
        float *f = static_cast<float *>(base);
        lu = f;
        int *i = reinterpret_cast<int *>(f + kCaluW * kCaluW);
        cand = i;
        gcand = cand + kCaluMaxCtas * kCaluW;
        gp = gcand + kCaluGroup * kCaluW;
        moves = gp + kCaluW;
        nmoves = moves + 4 * kCaluW;
        count = reinterpret_cast<unsigned *>(nmoves + 1);
    }
};

struct CaluShared {
    unsigned long long key[2][kCaluWarps];   // each warp's best candidate, by column parity
    __align__(16) float row[2][kCaluWarps][kCaluW];  // that candidate's row
    int sel[kCaluW];
    int last;
};

// Order of a live row as a pivot candidate: |v| above zero/NaN, then the
// lower row; 0 is reserved for "no candidate".
__device__ __forceinline__ unsigned long long calu_key(float v, int row) {
    const float m = fabsf(v);
    const unsigned hi = m > 0.f ? __float_as_uint(m) + 2u : 1u;
    return ((unsigned long long)hi << 32) | (unsigned)(~(unsigned)row);
}

__device__ __forceinline__ unsigned long long umax64(unsigned long long a, unsigned long long b) {
    return a > b ? a : b;
}

// The first w columns of row `row` from column c into a[] (zeros past w or
// for a dead row); vec: rows start on 16-byte boundaries.
__device__ __forceinline__ void calu_load_row(float (&a)[kCaluW], const float *A, int64_t lda,
                                              int row, int c, int w, bool live, bool vec) {
    const float *src = A + (int64_t)(live ? row : 0) * lda + c;
#pragma unroll
    for (int q = 0; q < kCaluW / 4; ++q) {
        float4 v = make_float4(0.f, 0.f, 0.f, 0.f);
        if (live) {
            if (vec && 4 * q + 4 <= w) {
                v = *reinterpret_cast<const float4 *>(src + 4 * q);
            } else if (4 * q + 4 <= w) {
                v.x = src[4 * q];
                v.y = src[4 * q + 1];
                v.z = src[4 * q + 2];
                v.w = src[4 * q + 3];
            } else if (4 * q < w) {
                v.x = src[4 * q];
                if (4 * q + 1 < w) v.y = src[4 * q + 1];
                if (4 * q + 2 < w) v.z = src[4 * q + 2];
            }
        }
        a[4 * q] = v.x;
        a[4 * q + 1] = v.y;
        a[4 * q + 2] = v.z;
        a[4 * q + 3] = v.w;
    }
}

// Partial pivoting over the CTA's rows (one per thread: a[] its first w
// columns, `row` its global index, dead threads live = false).  Picks up to w
// rows, their global indices in pick order into sh.sel, and returns how many.
// KEEP_L keeps the multipliers, so a picked row ends as its L\U row;
// picked_at = the column at which this thread's row was picked, else -1.
template <bool KEEP_L>
__device__ int calu_gepp(float (&a)[kCaluW], int row, bool live, int w, CaluShared &sh,
                         int &picked_at) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int np = 0;
    picked_at = -1;
#pragma unroll
    for (int j = 0; j < kCaluW; ++j) {
        if (j >= w) break;
        const int b = j & 1;
        const unsigned long long k = live ? calu_key(a[j], row) : 0ull;
        unsigned long long best = k;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) best = umax64(best, __shfl_xor_sync(0xffffffffu, best, o));
        if (lane == 0) sh.key[b][warp] = best;
        if (k != 0ull && k == best) {
            float4 *dst = reinterpret_cast<float4 *>(sh.row[b][warp]);
#pragma unroll
            for (int q = 0; q < kCaluW / 4; ++q)
                if (4 * q + 3 >= j)
                    dst[q] = make_float4(a[4 * q], a[4 * q + 1], a[4 * q + 2], a[4 * q + 3]);
        }
        __syncthreads();
        const unsigned long long mine = lane < kCaluWarps ? sh.key[b][lane] : 0ull;
        unsigned long long g = mine;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) g = umax64(g, __shfl_xor_sync(0xffffffffu, g, o));
        if (g == 0ull) break;  // no candidate left in the CTA (uniform)
        const int p = (int)(~(unsigned)(g & 0xffffffffull));
        const int ww = __ffs(__ballot_sync(0xffffffffu, mine == g)) - 1;
        const float *prow = sh.row[b][ww];
        float pv = prow[j];
        if (pv == 0.f) pv = pivot_floor<float>::value;
        const float rp = __frcp_rn(pv);
        if (live && row == p) {
            live = false;
            picked_at = j;
        }
        if (live) {
            const float l = a[j] * rp;
            if (KEEP_L) a[j] = l;
#pragma unroll
            for (int q = 0; q < kCaluW / 4; ++q) {
                if (4 * q + 3 > j) {
                    const float4 u = reinterpret_cast<const float4 *>(prow)[q];
                    if (4 * q > j) a[4 * q] = fmaf(-l, u.x, a[4 * q]);
                    if (4 * q + 1 > j) a[4 * q + 1] = fmaf(-l, u.y, a[4 * q + 1]);
                    if (4 * q + 2 > j) a[4 * q + 2] = fmaf(-l, u.z, a[4 * q + 2]);
                    a[4 * q + 3] = fmaf(-l, u.w, a[4 * q + 3]);
                }
            }
        }
        if (tid == 0) sh.sel[j] = p;
        np = j + 1;
    }
    __syncthreads();
    return np;
}

// Every thread's writes before, one arrival on *count after; true in the
// CTA whose arrival completes `members`.
__device__ __forceinline__ bool calu_arrive(unsigned *count, int members, CaluShared &sh) {
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) sh.last = atomicAdd(count, 1u) == (unsigned)(members - 1);
    __syncthreads();
    const bool last = sh.last != 0;
    if (last) __threadfence();
    return last;
}

// The final CTA: the pivot rows' L11\U11, the interchanges, the moves, info,
// and the counters back to zero.
__device__ void calu_finish(const float (&a)[kCaluW], int row, int picked, int np, int c, int w,
                            CaluScratch s, int32_t *ipiv, int32_t *info, CaluShared &sh) {
    const int tid = threadIdx.x, lane = tid & 31;
    // The row buffers are free after the last pivot search: 32 x 32 floats.
    float(*lus)[kCaluW] = reinterpret_cast<float(*)[kCaluW]>(&sh.row[0][0][0]);
    if (picked >= 0) {
        float4 *g = reinterpret_cast<float4 *>(s.lu + picked * kCaluW);
        float4 *l = reinterpret_cast<float4 *>(lus[picked]);
#pragma unroll
        for (int q = 0; q < kCaluW / 4; ++q) {
            const float4 v = make_float4(a[4 * q], a[4 * q + 1], a[4 * q + 2], a[4 * q + 3]);
            g[q] = v;
            l[q] = v;
        }
    }
    if (tid <= kCaluGroup) s.count[tid] = 0u;
    __syncthreads();
    if (tid >= 32) return;
    // LAPACK-style interchanges: step j swaps position c + j with the current
    // position of pivot j.  Lane k tracks position c + k and, from step k on,
    // possibly one more position outside [c, c + 32); untracked positions hold
    // their own rows.
    const unsigned full = 0xffffffffu;
    int pos0 = c + lane, row0 = c + lane, pos1 = -1, row1 = -1;
    for (int j = 0; j < np; ++j) {
        const int g = sh.sel[j], cj = c + j;
        int where = row0 == g ? pos0 : (row1 == g ? pos1 : -1);
        unsigned m = __ballot_sync(full, where >= 0);
        const int pos = m ? __shfl_sync(full, where, __ffs(m) - 1) : g;
        int here = pos0 == cj ? row0 : (pos1 == cj ? row1 : -1);
        m = __ballot_sync(full, here >= 0);
        const int at_cj = m ? __shfl_sync(full, here, __ffs(m) - 1) : cj;
        const bool tracked = __any_sync(full, pos0 == pos || pos1 == pos);
        if (pos0 == cj) row0 = g;
        else if (pos0 == pos) row0 = at_cj;
        if (pos1 == cj) row1 = g;
        else if (pos1 == pos) row1 = at_cj;
        if (!tracked && lane == j) {
            pos1 = pos;
            row1 = at_cj;
        }
        if (lane == 0) ipiv[cj] = pos;
    }
    const bool mv0 = row0 != pos0, mv1 = pos1 >= 0 && row1 != pos1;
    const unsigned b0 = __ballot_sync(full, mv0), b1 = __ballot_sync(full, mv1);
    const unsigned lt = (1u << lane) - 1u;
    if (mv0) {
        const int i = __popc(b0 & lt);
        s.moves[2 * i] = row0;
        s.moves[2 * i + 1] = pos0;
    }
    if (mv1) {
        const int i = __popc(b0) + __popc(b1 & lt);
        s.moves[2 * i] = row1;
        s.moves[2 * i + 1] = pos1;
    }
    s.gp[lane] = lane < np ? sh.sel[lane] : -1;
    const unsigned zero = __ballot_sync(full, lane < np && lus[lane][lane] == 0.f);
    if (lane == 0) {
        *s.nmoves = __popc(b0) + __popc(b1);
        if (zero && *info == 0) *info = c + __ffs(zero);
    }
}

// Pivot search of the leaf at column c (w <= 32 columns, rows [c, n)) over
// nctas CTAs of 512 rows.
__global__ void __launch_bounds__(kCaluRows)
    calu_pick_kernel(const float *A, int64_t lda, int n, int c, int w, int nctas, bool vec,
                     CaluScratch s, int32_t *ipiv, int32_t *info) {
    __shared__ CaluShared sh;
    const int tid = threadIdx.x;
    const int ngroups = (nctas + kCaluGroup - 1) / kCaluGroup;
    float a[kCaluW];
    int picked = -1;
    int row = c + blockIdx.x * kCaluRows + tid;
    bool live = row < n;
    calu_load_row(a, A, lda, row, c, w, live, vec);
    if (nctas == 1) {
        const int np = calu_gepp<true>(a, row, live, w, sh, picked);
        calu_finish(a, row, picked, np, c, w, s, ipiv, info, sh);
        return;
    }
    int np = calu_gepp<false>(a, row, live, w, sh, picked);
    if (tid < kCaluW) s.cand[blockIdx.x * kCaluW + tid] = tid < np ? sh.sel[tid] : -1;
    const int grp = blockIdx.x / kCaluGroup;
    const int members = min(kCaluGroup, nctas - grp * kCaluGroup);
    if (!calu_arrive(&s.count[grp], members, sh)) return;
    // Second level: the group's candidates, original values.
    row = tid < members * kCaluW ? __ldcg(&s.cand[grp * kCaluGroup * kCaluW + tid]) : -1;
    live = row >= 0;
    calu_load_row(a, A, lda, row, c, w, live, vec);
    if (ngroups == 1) {
        np = calu_gepp<true>(a, row, live, w, sh, picked);
        calu_finish(a, row, picked, np, c, w, s, ipiv, info, sh);
        return;
    }
    np = calu_gepp<false>(a, row, live, w, sh, picked);
    if (tid < kCaluW) s.gcand[grp * kCaluW + tid] = tid < np ? sh.sel[tid] : -1;
    if (!calu_arrive(&s.count[kCaluGroup], ngroups, sh)) return;
    // Third level: every group's candidates.
    row = tid < ngroups * kCaluW ? __ldcg(&s.gcand[tid]) : -1;
    live = row >= 0;
    calu_load_row(a, A, lda, row, c, w, live, vec);
    np = calu_gepp<true>(a, row, live, w, sh, picked);
    calu_finish(a, row, picked, np, c, w, s, ipiv, info, sh);
}

// After the pivot search: CTAs [0, panel_ctas) take the panel's rows, one
// per thread -- a pivot row's place c + j gets L11\U11 row j, every other
// row becomes l = a U11^-1 at its final position; the CTAs after them move
// the rows that change place in every column outside the panel (all reads
// of a column before its writes).  No row is read by one thread and written
// by another: displaced rows land on the pivots' old places, which their
// own threads leave alone.
__global__ void __launch_bounds__(kCaluApplyThreads)
    calu_apply_kernel(float *A, int64_t lda, int n, int c, int w, int panel_ctas, bool vec,
                      CaluScratch s) {
    __shared__ __align__(16) float U[kCaluW][kCaluW];
    __shared__ float rd[kCaluW];
    __shared__ int gp[kCaluW];
    __shared__ int mv[4 * kCaluW];
    __shared__ int nmv;
    const int tid = threadIdx.x;
    for (int e = tid; e < kCaluW * kCaluW; e += kCaluApplyThreads) (&U[0][0])[e] = s.lu[e];
    for (int e = tid; e < 4 * kCaluW; e += kCaluApplyThreads) mv[e] = s.moves[e];
    if (tid < kCaluW) gp[tid] = s.gp[tid];
    if (tid == 0) nmv = *s.nmoves;
    __syncthreads();
    if (tid < kCaluW) {
        float d = U[tid][tid];
        if (d == 0.f) d = pivot_floor<float>::value;
        rd[tid] = __frcp_rn(d);
    }
    __syncthreads();
    const int nm = nmv;
    if ((int)blockIdx.x < panel_ctas) {
        const int row = c + blockIdx.x * kCaluApplyThreads + tid;
        if (row >= n) return;
        bool pivot = false;
#pragma unroll 8
        for (int k = 0; k < kCaluW; ++k) pivot |= gp[k] == row;
        float x[kCaluW];
        int dst = row;
        if (!pivot) {
            if (row < c + kCaluW)
                for (int k = 0; k < nm; ++k)
                    if (mv[2 * k] == row) dst = mv[2 * k + 1];
            calu_load_row(x, A, lda, row, c, w, true, vec);
#pragma unroll
            for (int j = 0; j < kCaluW; ++j) {
                if (j < w) {
                    const float l = x[j] * rd[j];
                    x[j] = l;
#pragma unroll
                    for (int q = 0; q < kCaluW / 4; ++q) {
                        if (4 * q + 3 > j) {
                            const float4 u = reinterpret_cast<const float4 *>(U[j])[q];
                            if (4 * q > j) x[4 * q] = fmaf(-l, u.x, x[4 * q]);
                            if (4 * q + 1 > j) x[4 * q + 1] = fmaf(-l, u.y, x[4 * q + 1]);
                            if (4 * q + 2 > j) x[4 * q + 2] = fmaf(-l, u.z, x[4 * q + 2]);
                            x[4 * q + 3] = fmaf(-l, u.w, x[4 * q + 3]);
                        }
                    }
                }
            }
            float *out = A + (int64_t)dst * lda + c;
#pragma unroll
            for (int j = 0; j < kCaluW; ++j)
                if (j < w) out[j] = x[j];
        }
        // Row c + k (k < w) ends holding pivot k's L\U row.
        if (row < c + w) {
            const int k = row - c;
            float *out = A + (int64_t)row * lda + c;
            for (int j = 0; j < w; ++j) out[j] = U[k][j];
        }
        return;
    }
    const int col = (blockIdx.x - panel_ctas) * kCaluApplyThreads + tid;
    if (col >= n || (col >= c && col < c + w)) return;
    float v[2 * kCaluW];
#pragma unroll
    for (int k = 0; k < 2 * kCaluW; ++k)
        if (k < nm) v[k] = A[(int64_t)mv[2 * k] * lda + col];
#pragma unroll
    for (int k = 0; k < 2 * kCaluW; ++k)
        if (k < nm) A[(int64_t)mv[2 * k + 1] * lda + col] = v[k];
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
template <typename T, bool UNIT>
__global__ void trsm_lower_leaf_kernel(const T *A, int64_t lda, int r, int w, T *B, int64_t ldb,
                                       int c0, int c1) {
    __shared__ T Ls[kTrsmLeaf][kTrsmLeaf + 1];
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
        int i = e / w, j = e - i * w;
        Ls[i][j] = A[(int64_t)(r + i) * lda + r + j];
    }
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
    for (int e = threadIdx.x; e < w * w; e += blockDim.x) {
        int i = e / w, j = e - i * w;
        T v = A[(int64_t)(r + i) * lda + r + j];
        if (TRANS)
            Us[j][i] = v;
        else
            Us[i][j] = v;
    }
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

// Tournament-pivoting leaf: the pivot search, then the rows into place.
static int calu_leaf(LuRun<float> &R, int c, int w) {
    const int m = R.n - c;
    const int nctas = (int)ceil_div(m, kCaluRows);
    const bool vec = R.lda % 4 == 0 && reinterpret_cast<uintptr_t>(R.A) % 16 == 0;
    calu_pick_kernel<<<nctas, kCaluRows, 0, R.st>>>(R.A, R.lda, R.n, c, w, nctas, vec, R.cs,
                                                    R.ipiv, R.info);
    const int panel = (int)ceil_div(m, kCaluApplyThreads);
    const int other = (int)ceil_div(R.n, kCaluApplyThreads);
    calu_apply_kernel<<<panel + other, kCaluApplyThreads, 0, R.st>>>(R.A, R.lda, R.n, c, w, panel,
                                                                     vec, R.cs);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

template <typename T>
static int leaf(LuRun<T> &R, int c, int w) {
    const int m = R.n - c;
    const int threads = 256;
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
        laswp_kernel<T><<<(unsigned)ceil_div(R.n, threads), threads, 0, R.st>>>(
            R.A, R.lda, R.n, c, w, R.ipiv, c, c + w);
        NMX_CUDA_TRY(cudaGetLastError());
        return 0;
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
    // The interchanges across the rest of the width.
    laswp_kernel<T><<<(unsigned)ceil_div(R.n, threads), threads, 0, R.st>>>(R.A, R.lda, R.n, c, w,
                                                                             R.ipiv, c, c + w);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

// X := L^-1 X, L the w x w lower block at (r, r) of A, X rows [r, r+w) cols [c0, c1) of B.
template <typename T, bool UNIT>
int trsm_lower(const GemmSub &gs, const T *A, int64_t lda, int r, int w, T *B, int64_t ldb, int c0,
               int c1) {
    cudaStream_t st = gs.st;
    if (w <= 0 || c1 <= c0) return 0;
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
    cublasHandle_t h = gs.h;
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
    // B_top -= U_top,bot X_bot   (TRANS: U_top,bot = (L_bot,top)^T)
    if (TRANS) {
        const T minus = T(-1), one = T(1);
        // row-major C[hw x nc] -= (L[bot x top])^T X[bot x nc]; column-major: C^T -= X^T L
        cublasStatus_t s;
        if (sizeof(T) == 8)
            s = cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, c1 - c0, hw, w - hw, (const double *)&minus,
                            (const double *)(B + (int64_t)(r + hw) * ldb + c0), (int)ldb,
                            (const double *)(A + (int64_t)(r + hw) * lda + r), (int)lda,
                            (const double *)&one, (double *)(B + (int64_t)r * ldb + c0), (int)ldb);
        else
            s = cublasSgemm(h, CUBLAS_OP_N, CUBLAS_OP_T, c1 - c0, hw, w - hw, (const float *)&minus,
                            (const float *)(B + (int64_t)(r + hw) * ldb + c0), (int)ldb,
                            (const float *)(A + (int64_t)(r + hw) * lda + r), (int)lda,
                            (const float *)&one, (float *)(B + (int64_t)r * ldb + c0), (int)ldb);
        NMX_CUBLAS_TRY(s);
    } else {
        rc = gs(hw, c1 - c0, w - hw, A + (int64_t)r * lda + r + hw, lda,
                B + (int64_t)(r + hw) * ldb + c0, ldb, B + (int64_t)r * ldb + c0, ldb);
        if (rc) return rc;
    }
    return trsm_upper<T, TRANS>(gs, A, lda, r, hw, B, ldb, c0, c1);
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
    rc = trsm_lower<T, true>(R.gs, R.A, R.lda, c, hw, R.A, R.lda, c + hw, c + w);
    if (rc) return rc;
    // A22 -= L21 U12.
    rc = R.gs(R.n - c - hw, w - hw, hw, R.A + (int64_t)(c + hw) * R.lda + c, R.lda,
              R.A + (int64_t)c * R.lda + c + hw, R.lda, R.A + (int64_t)(c + hw) * R.lda + c + hw,
              R.lda);
    if (rc) return rc;
    return getrf2<T>(R, c + hw, w - hw);
}

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
    // Tournament pivoting: FP32 panels of up to 131072 rows.
    if (std::is_same<T, float>::value && tournament && n <= (int64_t)kCaluMaxCtas * kCaluRows) {
        void *cv = nullptr;
        rc = ctx->ensure_slot(kWsCalu, CaluScratch::bytes(), &cv);
        if (rc) return rc;
        R.cs.carve(cv);
        NMX_CUDA_TRY(cudaMemsetAsync(R.cs.count, 0, sizeof(unsigned) * (kCaluGroup + 1), st));
        R.tournament = true;
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
    int rc = ctx_cublas(ctx, gs.st, &gs.h);
    if (rc) return rc;
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
    int rc = ctx_cublas(ctx, st, &gs.h);
    if (rc) return rc;
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
