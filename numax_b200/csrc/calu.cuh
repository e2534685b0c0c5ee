// LU panel kernels (dense_lu.cu): the tournament-pivoting (CALU) leaf and
// the one-kernel panel TRSM of the FP32 factorization, and the row-move
// kernels that carry any leaf's interchanges to the other columns.
#pragma once

#include <cstddef>
#include <cstdint>

#include "nmx_common.cuh"

namespace nmx {

// ---- tournament-pivoting leaf (FP32: the mixed-precision factorization) ----
//
// The FP32 factorization inside iterative refinement (ir.cu) needs a stable
// LU, not numax's exact pivot sequence: refinement in FP64 makes the solution
// independent of which stable pivots the factors used.  Its leaves use
// tournament pivoting (CALU; Grigori, Demmel & Xiang, SIAM J. Matrix Anal.
// Appl. 32(4), 2011) over a reduction tree of at most three levels:
//   1. every CTA holds 512 rows of the panel, two rows per thread in
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
// independent), puts the panel's rows in their final places and, in extra
// CTAs, moves the same rows in the other columns in scope.  The pivot search
// costs one CTA barrier per column instead of one grid- or cluster-wide
// exchange.  A zero U11 diagonal is floored to 1e-30
// and the first one reported in info; a column without a nonzero candidate
// picks the lowest row.
constexpr int kCaluRows = 512;                          // rows per CTA
constexpr int kCaluThreads = 256;                       // two rows per thread
constexpr int kCaluW = 32;                              // widest leaf
constexpr int kCaluWarps = kCaluThreads / 32;
constexpr int kCaluGroup = kCaluRows / kCaluW;          // candidate sets one CTA stacks
constexpr int kCaluMaxCtas = kCaluGroup * kCaluGroup;   // panels of up to 131072 rows
constexpr int kCaluApplyThreads = 256;
// A leaf's row moves: the count, then up to 2 kCaluW (from, to) row pairs.
constexpr int kCaluListStride = 1 + 4 * kCaluW;
// Leaves of one look-ahead panel: <= 2048 columns of tournament leaves, <= 512
// of partial-pivoting leaves (which can be as narrow as 8 columns).
constexpr int kCaluMaxLists = 64;

struct CaluScratch {
    int *cand;        // [kCaluMaxCtas][kCaluW] first-level picks (global rows, -1: none)
    int *gcand;       // [kCaluGroup][kCaluW] second-level picks
    unsigned *count;  // [kCaluGroup + 1] arrival counters, zero between leaves
    float *lu;        // [kCaluW][kCaluW] L11\U11 of the pivot rows, pivot order
    float *lmul;      // [kCaluW][kCaluRows] the final CTA's multipliers, step-major
    int *gp;          // [kCaluW] pivot rows in pivot order (-1 past the panel)
    int *lists;       // [2][kCaluMaxLists][kCaluListStride] the leaves' row moves
    static size_t bytes() {
        return sizeof(int) * ((size_t)kCaluMaxCtas * kCaluW + kCaluGroup * kCaluW + kCaluGroup +
                              1 + kCaluW + 2 * kCaluMaxLists * kCaluListStride) +
               sizeof(float) * (kCaluW * kCaluW + kCaluW * kCaluRows) + 256;
    }
    void carve(void *base) {
        float *f = static_cast<float *>(base);
        lu = f;
        lmul = lu + kCaluW * kCaluW;
        int *i = reinterpret_cast<int *>(lmul + kCaluW * kCaluRows);
        cand = i;
        gcand = cand + kCaluMaxCtas * kCaluW;
        gp = gcand + kCaluGroup * kCaluW;
        lists = gp + kCaluW;
        count = reinterpret_cast<unsigned *>(lists + 2 * kCaluMaxLists * kCaluListStride);
    }
};

struct CaluShared {
    unsigned key[2][kCaluWarps];   // each warp's best candidate, by column parity
    int rid[2][kCaluWarps];        // its global row
    __align__(16) float row[2][kCaluWarps][kCaluW];  // its row
    int sel[kCaluW];
    int ipv[kCaluW];
    int zdiag[kCaluW];
    int last;
};

// A thread's two rows: slot 0 is CTA row tid, slot 1 is CTA row tid + 256.
struct CaluRows {
    float a[2][kCaluW];
    int row[2];
    bool live[2];
    int picked[2];  // the step that picked the row, or -1
};

// Order of a row as a pivot candidate: |v| above zero/NaN, then slot 0 (the
// lower rows); 0 is "no candidate".  Within a slot, the lower lane and the
// lower warp win ties, so in a CTA's own rows the first maximum wins, as in
// partial pivoting.
__device__ __forceinline__ unsigned calu_key(float v, int slot) {
    const float m = fabsf(v);
    const unsigned hi = m > 0.f ? __float_as_uint(m) + 2u : 1u;
    return (hi << 1) | (slot == 0 ? 1u : 0u);
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

__device__ __forceinline__ void calu_load(CaluRows &R, const float *A, int64_t lda, int row0,
                                          int row1, int c, int w, bool vec) {
    R.row[0] = row0;
    R.row[1] = row1;
    R.live[0] = row0 >= 0;
    R.live[1] = row1 >= 0;
    calu_load_row(R.a[0], A, lda, row0, c, w, R.live[0], vec);
    calu_load_row(R.a[1], A, lda, row1, c, w, R.live[1], vec);
}

__device__ __forceinline__ void calu_put_row(float *dst, const float (&a)[kCaluW]) {
    float4 *d = reinterpret_cast<float4 *>(dst);
#pragma unroll
    for (int q = 0; q < kCaluW / 4; ++q)
        d[q] = make_float4(a[4 * q], a[4 * q + 1], a[4 * q + 2], a[4 * q + 3]);
}

// a := a shifted left by one column minus l times the pivot row likewise.
__device__ __forceinline__ void calu_eliminate(float (&a)[kCaluW], float l, const float4 *prow) {
    float4 u = prow[0];
    a[0] = fmaf(-l, u.y, a[1]);
    a[1] = fmaf(-l, u.z, a[2]);
    a[2] = fmaf(-l, u.w, a[3]);
#pragma unroll
    for (int q = 1; q < kCaluW / 4; ++q) {
        u = prow[q];
        a[4 * q - 1] = fmaf(-l, u.x, a[4 * q]);
        a[4 * q] = fmaf(-l, u.y, a[4 * q + 1]);
        a[4 * q + 1] = fmaf(-l, u.z, a[4 * q + 2]);
        a[4 * q + 2] = fmaf(-l, u.w, a[4 * q + 3]);
    }
    a[kCaluW - 1] = 0.f;
}

// Partial pivoting over the CTA's rows (two per thread).  Picks up to w
// rows, their global indices in pick order into sh.sel, and returns how many.
// Every live row shifts left by one column per step, so the column being
// eliminated is always a[0] and the loop body is the same for every column.
// A row picked at step j stops there: its a[0..31-j] hold its U row from
// column j on.  lmul (non-null) receives every live row's multiplier at
// every step, [j][slot * 256 + tid].
__device__ int calu_gepp(CaluRows &R, int w, CaluShared &sh, float *lmul) {
    const unsigned full = 0xffffffffu;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    int np = 0;
    R.picked[0] = R.picked[1] = -1;
#pragma unroll 1
    for (int j = 0; j < w; ++j) {
        const int b = j & 1;
        const unsigned k0 = R.live[0] ? calu_key(R.a[0][0], 0) : 0u;
        const unsigned k1 = R.live[1] ? calu_key(R.a[1][0], 1) : 0u;
        const unsigned mine = k0 > k1 ? k0 : k1;
        const unsigned wk = __reduce_max_sync(full, mine);
        const int wl = __ffs(__ballot_sync(full, mine == wk)) - 1;
        if (lane == wl) {
            sh.key[b][warp] = wk;
            const bool first = k0 == wk;
            sh.rid[b][warp] = first ? R.row[0] : R.row[1];
            if (wk != 0u) {
                if (first) calu_put_row(sh.row[b][warp], R.a[0]);
                else calu_put_row(sh.row[b][warp], R.a[1]);
            }
        }
        __syncthreads();
        const unsigned mk = lane < kCaluWarps ? sh.key[b][lane] : 0u;
        const unsigned gk = __reduce_max_sync(full, mk);
        if (gk == 0u) break;  // no candidate left in the CTA (uniform)
        const int ww = __ffs(__ballot_sync(full, mk == gk)) - 1;
        const int p = sh.rid[b][ww];
        const float4 *prow = reinterpret_cast<const float4 *>(sh.row[b][ww]);
        const float pv = sh.row[b][ww][0];
        const float rp = __fdividef(1.0f, pv == 0.f ? pivot_floor<float>::value : pv);
#pragma unroll
        for (int s = 0; s < 2; ++s) {
            if (R.live[s] && R.row[s] == p) {
                R.live[s] = false;
                R.picked[s] = j;
            }
            if (R.live[s]) {
                const float l = R.a[s][0] * rp;
                if (lmul) lmul[j * kCaluRows + s * kCaluThreads + tid] = l;
                calu_eliminate(R.a[s], l, prow);
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

// The final CTA: the pivot rows' L11\U11, the interchanges, the row moves
// (into mlist), info, and the counters back to zero.  A picked row holds its
// U row in a[] and its multipliers in s.lmul.
__device__ void calu_finish(const CaluRows &R, int np, int c, CaluScratch s, int32_t *ipiv,
                            int32_t *info, int *mlist, CaluShared &sh) {
    const int tid = threadIdx.x, lane = tid & 31;
#pragma unroll
    for (int sl = 0; sl < 2; ++sl) {
        const int pk = R.picked[sl];
        if (pk >= 0) {
            float *dst = s.lu + pk * kCaluW;
            const float *lm = s.lmul + sl * kCaluThreads + tid;
            float l[kCaluW];
#pragma unroll
            for (int k = 0; k < kCaluW; ++k) l[k] = k < pk ? lm[k * kCaluRows] : 0.f;
#pragma unroll
            for (int k = 0; k < kCaluW; ++k)
                if (k < pk) dst[k] = l[k];
#pragma unroll
            for (int i = 0; i < kCaluW; ++i)
                if (pk + i < kCaluW) dst[pk + i] = R.a[sl][i];
            sh.zdiag[pk] = R.a[sl][0] == 0.f;
        }
    }
    if (tid <= kCaluGroup) s.count[tid] = 0u;
    __syncthreads();
    if (tid >= 32) return;
    // LAPACK-style interchanges: step j swaps position c + j with the current
    // position of pivot j.  A row moves at step i exactly when it sits at
    // c + i then, and goes to ipiv[i] > c + i; so pivot j's position is found
    // by following ipiv from its own row while the position is below c + j.
    if (lane == 0) {
        for (int j = 0; j < np; ++j) {
            int pos = sh.sel[j];
            while (pos - c < j) pos = sh.ipv[pos - c];
            sh.ipv[j] = pos;
            ipiv[c + j] = pos;
        }
    }
    __syncwarp();
    // Moves: pivot j to c + j, and every other row of [c, c + np) to the end
    // of its chain.
    const unsigned full = 0xffffffffu;
    const int r = c + lane;
    bool pivot = false;
    for (int j = 0; j < np; ++j) pivot |= sh.sel[j] == r;
    int to = r;
    if (!pivot && lane < np) {
        to = sh.ipv[lane];
        while (to - c < np) to = sh.ipv[to - c];
    }
    const int g = lane < np ? sh.sel[lane] : -1;
    const bool mv0 = g >= 0 && g != r, mv1 = to != r;
    const unsigned b0 = __ballot_sync(full, mv0), b1 = __ballot_sync(full, mv1);
    const unsigned lt = (1u << lane) - 1u;
    if (mv0) {
        const int i = __popc(b0 & lt);
        mlist[1 + 2 * i] = g;
        mlist[2 + 2 * i] = r;
    }
    if (mv1) {
        const int i = __popc(b0) + __popc(b1 & lt);
        mlist[1 + 2 * i] = r;
        mlist[2 + 2 * i] = to;
    }
    s.gp[lane] = g;
    const unsigned zero = __ballot_sync(full, lane < np && sh.zdiag[lane] != 0);
    if (lane == 0) {
        mlist[0] = __popc(b0) + __popc(b1);
        if (zero && *info == 0) *info = c + __ffs(zero);
    }
}

// Pivot search of the leaf at column c (w <= 32 columns, rows [c, n)) over
// nctas CTAs of 512 rows.
__global__ void __launch_bounds__(kCaluThreads)
    calu_pick_kernel(const float *A, int64_t lda, int n, int c, int w, int nctas, bool vec,
                     CaluScratch s, int32_t *ipiv, int32_t *info, int *mlist) {
    __shared__ CaluShared sh;
    const int tid = threadIdx.x;
    const int ngroups = (nctas + kCaluGroup - 1) / kCaluGroup;
    CaluRows R;
    {
        const int r0 = c + blockIdx.x * kCaluRows + tid, r1 = r0 + kCaluThreads;
        calu_load(R, A, lda, r0 < n ? r0 : -1, r1 < n ? r1 : -1, c, w, vec);
    }
    if (nctas == 1) {
        const int np = calu_gepp(R, w, sh, s.lmul);
        calu_finish(R, np, c, s, ipiv, info, mlist, sh);
        return;
    }
    int np = calu_gepp(R, w, sh, nullptr);
    if (tid < kCaluW) s.cand[blockIdx.x * kCaluW + tid] = tid < np ? sh.sel[tid] : -1;
    const int grp = blockIdx.x / kCaluGroup;
    const int members = min(kCaluGroup, nctas - grp * kCaluGroup);
    if (!calu_arrive(&s.count[grp], members, sh)) return;
    // Second level: the group's candidates, original values.
    {
        const int *gc = s.cand + grp * kCaluGroup * kCaluW;
        const int k1 = tid + kCaluThreads, lim = members * kCaluW;
        calu_load(R, A, lda, tid < lim ? __ldcg(gc + tid) : -1, k1 < lim ? __ldcg(gc + k1) : -1, c,
                  w, vec);
    }
    if (ngroups == 1) {
        np = calu_gepp(R, w, sh, s.lmul);
        calu_finish(R, np, c, s, ipiv, info, mlist, sh);
        return;
    }
    np = calu_gepp(R, w, sh, nullptr);
    if (tid < kCaluW) s.gcand[grp * kCaluW + tid] = tid < np ? sh.sel[tid] : -1;
    if (!calu_arrive(&s.count[kCaluGroup], ngroups, sh)) return;
    // Third level: every group's candidates.
    {
        const int k1 = tid + kCaluThreads, lim = ngroups * kCaluW;
        calu_load(R, A, lda, tid < lim ? __ldcg(s.gcand + tid) : -1,
                  k1 < lim ? __ldcg(s.gcand + k1) : -1, c, w, vec);
    }
    np = calu_gepp(R, w, sh, s.lmul);
    calu_finish(R, np, c, s, ipiv, info, mlist, sh);
}

// Row moves in columns [a0, a1) and [b0, b1), a column per thread (CTA
// `cta` of the ones covering them): the lists in order, each list's reads of
// a column before its writes.  (Any LU leaf's interchanges: the tournament
// leaves write their lists, the partial-pivoting leaves get theirs from
// ipiv_moves_kernel.)  from/to/nmv: shared scratch.
template <typename T>
__device__ __forceinline__ void calu_swap_cta(T *__restrict__ A, int64_t lda, const int *lists,
                                              int nlists, int a0, int a1, int b0, int b1, int cta,
                                              int64_t *from, int64_t *to, int *nmv) {
    const int tid = threadIdx.x;
    const int t = cta * kCaluApplyThreads + tid;
    const int na = a1 - a0;
    const int col = t < na ? a0 + t : b0 + (t - na);
    const bool mine = t < na || col < b1;
    for (int l = 0; l < nlists; ++l) {
        const int *ml = lists + (size_t)l * kCaluListStride;
        __syncthreads();
        if (tid < 2 * kCaluW) {
            from[tid] = (int64_t)ml[1 + 2 * tid] * lda;
            to[tid] = (int64_t)ml[2 + 2 * tid] * lda;
        }
        if (tid == 0) *nmv = ml[0];
        __syncthreads();
        if (!mine) continue;
        const int nm = *nmv;
        T v[2 * kCaluW];
#pragma unroll
        for (int k = 0; k < 2 * kCaluW; ++k)
            if (k < nm) v[k] = A[from[k] + col];
#pragma unroll
        for (int k = 0; k < 2 * kCaluW; ++k)
            if (k < nm) A[to[k] + col] = v[k];
    }
}

template <typename T>
__global__ void __launch_bounds__(kCaluApplyThreads)
    calu_swap_kernel(T *__restrict__ A, int64_t lda, const int *lists, int nlists, int a0, int a1,
                     int b0, int b1) {
    __shared__ int64_t from[2 * kCaluW], to[2 * kCaluW];
    __shared__ int nmv;
    calu_swap_cta<T>(A, lda, lists, nlists, a0, a1, b0, b1, blockIdx.x, from, to, &nmv);
}

// After the pivot search: 256 rows of the panel per CTA, staged through
// shared memory so global accesses are whole rows.  A pivot row is skipped
// (its place c + j gets L11\U11 row j), every other row becomes
// l = a U11^-1 at its final position.  No row is read by one CTA and written
// by another: displaced rows land on the pivots' old places, which their own
// CTAs leave alone, and rows c .. c+w-1 are read and written by CTA 0 alone.
// CTAs past panel_ctas move the leaf's rows in the other columns in scope,
// [a0, a1) and [b0, b1) (disjoint from the panel's columns).
constexpr int kCaluApplyPitch = kCaluW + 1;
constexpr size_t kCaluApplySmem = sizeof(float) * kCaluApplyThreads * kCaluApplyPitch;

__global__ void __launch_bounds__(kCaluApplyThreads)
    calu_apply_kernel(float *A, int64_t lda, int n, int c, int w, CaluScratch s,
                      const int *mlist, int panel_ctas, int a0, int a1, int b0, int b1) {
    __shared__ __align__(16) float U[kCaluW][kCaluW];
    __shared__ float rd[kCaluW];
    __shared__ int gp[kCaluW];
    __shared__ int mv[4 * kCaluW];
    __shared__ int dst[kCaluApplyThreads];
    __shared__ int nmv;
    extern __shared__ __align__(16) float tile[];  // [256][33] the CTA's rows
    __shared__ int64_t mfrom[2 * kCaluW], mto[2 * kCaluW];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if ((int)blockIdx.x >= panel_ctas) {
        calu_swap_cta<float>(A, lda, mlist, 1, a0, a1, b0, b1, (int)blockIdx.x - panel_ctas, mfrom,
                             mto, &nmv);
        return;
    }
    for (int e = tid; e < 4 * kCaluW; e += kCaluApplyThreads) mv[e] = mlist[1 + e];
    for (int e = tid; e < kCaluW * kCaluW; e += kCaluApplyThreads) (&U[0][0])[e] = s.lu[e];
    if (tid < kCaluW) gp[tid] = s.gp[tid];
    if (tid == 0) nmv = mlist[0];
    const int r0 = c + blockIdx.x * kCaluApplyThreads;
    const int nrows = min(kCaluApplyThreads, n - r0);
    // The CTA's rows into the tile, a warp per row, lanes over columns, eight
    // rows' loads in flight per warp.
    constexpr int NW = kCaluApplyThreads / 32;
#pragma unroll
    for (int r8 = 0; r8 < kCaluApplyThreads / NW; r8 += 8) {
        float v[8];
#pragma unroll
        for (int u = 0; u < 8; ++u) {
            const int r = warp + NW * (r8 + u);
            v[u] = (r < nrows && lane < w) ? A[(int64_t)(r0 + r) * lda + c + lane] : 0.f;
        }
#pragma unroll
        for (int u = 0; u < 8; ++u) tile[(warp + NW * (r8 + u)) * kCaluApplyPitch + lane] = v[u];
    }
    __syncthreads();
    if (tid < kCaluW) {
        float d = U[tid][tid];
        if (d == 0.f) d = pivot_floor<float>::value;
        rd[tid] = __frcp_rn(d);
    }
    const int nm = nmv;
    const int row = r0 + tid;
    int to = -1;
    if (tid < nrows) {
        bool pivot = false;
#pragma unroll 8
        for (int k = 0; k < kCaluW; ++k) pivot |= gp[k] == row;
        if (!pivot) {
            to = row;
            if (row < c + kCaluW)
                for (int k = 0; k < nm; ++k)
                    if (mv[2 * k] == row) to = mv[2 * k + 1];
        }
    }
    dst[tid] = to;
    __syncthreads();
    if (to >= 0) {
        float *t = tile + tid * kCaluApplyPitch;
        float x[kCaluW];
#pragma unroll
        for (int j = 0; j < kCaluW; ++j) x[j] = t[j];
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
#pragma unroll
        for (int j = 0; j < kCaluW; ++j) t[j] = x[j];
    }
    __syncthreads();
#pragma unroll 8
    for (int k = 0; k < kCaluApplyThreads / NW; ++k) {
        const int r = warp + NW * k;
        const int d = r < nrows ? dst[r] : -1;
        if (d >= 0 && lane < w) A[(int64_t)d * lda + c + lane] = tile[r * kCaluApplyPitch + lane];
    }
    // Rows c .. c+w-1: the pivots' L11\U11 (CTA 0, after its reads above).
    if (blockIdx.x == 0)
        for (int r = warp; r < w; r += kCaluApplyThreads / 32)
            if (lane < w) A[(int64_t)(c + r) * lda + c + lane] = U[r][lane];
}

// X := L^-1 X for the unit lower w x w block L at (r, r) of A (w <= 256, a
// multiple of 32) and X = rows [r, r + w) x columns [c0, c1) of B: the
// triangular solves of the tournament LU's panels in one kernel, a CTA per
// 32 columns with X in shared memory.  Warp b inverts the 32 x 32 diagonal
// block b by forward substitution (lane j forms column j), so each block step
// is two small products from shared memory: X_b := inv(L_bb) X_b, then
// X_below -= L_below,b X_b.
constexpr int kTrsmMaxW = 256;
constexpr int kTrsmThreads = 256;
constexpr int kTrsmXPitch = 33;
constexpr int kTrsmLPitch = 36;  // 16-byte rows for float4 reads
__host__ __device__ constexpr size_t trsm_unit_lower_smem(int w) {
    return sizeof(float) * ((size_t)w * kTrsmXPitch * 2 + (size_t)(w - 32) * kTrsmLPitch);
}

__global__ void __launch_bounds__(kTrsmThreads)
    trsm_unit_lower_kernel(const float *A, int64_t lda, int r, int w, float *B, int64_t ldb,
                           int c0, int c1) {
    extern __shared__ __align__(16) float tsm[];
    float *X = tsm;                          // [w][33] the CTA's 32 columns of X
    float *Li = X + w * kTrsmXPitch;         // [w/32][32][33] inverted diagonal blocks
    float *Ls = Li + w * kTrsmXPitch;        // [w-32][36] L below the current block
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = kTrsmThreads / 32;
    const int nb = w / 32;
    const int col = c0 + blockIdx.x * 32 + lane;
    const bool cv = col < c1;
    for (int i = warp; i < w; i += NW) X[i * kTrsmXPitch + lane] = cv ? B[(int64_t)(r + i) * ldb + col] : 0.f;
    if (warp < nb) {
        float *D = Li + warp * 32 * kTrsmXPitch;
        const int rb = r + 32 * warp;
        for (int i = 0; i < 32; ++i) D[i * kTrsmXPitch + lane] = A[(int64_t)(rb + i) * lda + rb + lane];
        __syncwarp();
        float x[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            float t = 0.f;
#pragma unroll
            for (int p = 0; p < i; ++p) t = fmaf(D[i * kTrsmXPitch + p], x[p], t);
            x[i] = i == lane ? 1.f : (i < lane ? 0.f : -t);
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 32; ++i) D[i * kTrsmXPitch + lane] = x[i];
    }
    __syncthreads();
    for (int b = 0; b < nb; ++b) {
        const int rb = 32 * b, below = w - rb - 32;
        for (int i = warp; i < below; i += NW)
            Ls[i * kTrsmLPitch + lane] = A[(int64_t)(r + rb + 32 + i) * lda + r + rb + lane];
        {
            const float *D = Li + b * 32 * kTrsmXPitch;
            float y[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll 8
            for (int p = 0; p < 32; ++p) {
                const float xp = X[(rb + p) * kTrsmXPitch + lane];
#pragma unroll
                for (int q = 0; q < 4; ++q) y[q] = fmaf(D[(4 * warp + q) * kTrsmXPitch + p], xp, y[q]);
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 4; ++q) X[(rb + 4 * warp + q) * kTrsmXPitch + lane] = y[q];
        }
        __syncthreads();
        if (below > 0) {
            float xb[32];
#pragma unroll
            for (int p = 0; p < 32; ++p) xb[p] = X[(rb + p) * kTrsmXPitch + lane];
            for (int i = warp; i < below; i += NW) {
                const float4 *lr = reinterpret_cast<const float4 *>(Ls + i * kTrsmLPitch);
                float t = 0.f;
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const float4 l = lr[q];
                    t = fmaf(l.x, xb[4 * q], t);
                    t = fmaf(l.y, xb[4 * q + 1], t);
                    t = fmaf(l.z, xb[4 * q + 2], t);
                    t = fmaf(l.w, xb[4 * q + 3], t);
                }
                X[(rb + 32 + i) * kTrsmXPitch + lane] -= t;
            }
        }
        __syncthreads();
    }
    if (cv)
        for (int i = warp; i < w; i += NW) B[(int64_t)(r + i) * ldb + col] = X[i * kTrsmXPitch + lane];
}

// The same solve for FP64 (and any T): X := L^-1 X for the unit lower w x w
// block (w <= 256, a multiple of 32), a CTA per 32 columns.  Every copy into
// shared memory goes by cp.async (the CTA's X, the diagonal blocks, and per
// block step the rows of L below it), so each is one round trip.
constexpr int kTrsmTPitchX = 33;
constexpr int kTrsmTPitchL = 33;
template <typename T>
__host__ __device__ constexpr size_t trsm_unit_lower_t_smem(int w) {
    return sizeof(T) * ((size_t)w * kTrsmTPitchX * 2 + (size_t)(w - 32) * kTrsmTPitchL);
}

template <typename T>
__device__ __forceinline__ void trsm_copy_async(T *dst, const T *src, bool ok) {
    const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
    if constexpr (sizeof(T) == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(d), "l"(src),
                     "r"(ok ? 8 : 0)
                     : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(d), "l"(src),
                     "r"(ok ? 4 : 0)
                     : "memory");
}

template <typename T>
__global__ void __launch_bounds__(kTrsmThreads)
    trsm_unit_lower_t_kernel(const T *A, int64_t lda, int r, int w, T *B, int64_t ldb, int c0,
                             int c1) {
    extern __shared__ __align__(16) unsigned char tsm_raw[];
    T *X = reinterpret_cast<T *>(tsm_raw);  // [w][33] the CTA's 32 columns of X
    T *Li = X + w * kTrsmTPitchX;             // [w/32][32][33] inverted diagonal blocks
    T *Ls = Li + w * kTrsmTPitchX;            // [w-32][33] L below the current block
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    constexpr int NW = kTrsmThreads / 32;
    const int nb = w / 32;
    const int col = c0 + blockIdx.x * 32 + lane;
    const bool cv = col < c1;
    for (int i = warp; i < w; i += NW)
        trsm_copy_async(&X[i * kTrsmTPitchX + lane], cv ? &B[(int64_t)(r + i) * ldb + col] : B, cv);
    if (warp < nb) {
        const int rb = r + 32 * warp;
        T *D = Li + warp * 32 * kTrsmTPitchX;
        for (int i = 0; i < 32; ++i)
            trsm_copy_async(&D[i * kTrsmTPitchX + lane], &A[(int64_t)(rb + i) * lda + rb + lane], true);
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    if (warp < nb) {
        // Lane j forms column j of the inverse by forward substitution.
        T *D = Li + warp * 32 * kTrsmTPitchX;
        T x[32];
#pragma unroll
        for (int i = 0; i < 32; ++i) {
            T t = T(0);
#pragma unroll
            for (int p = 0; p < i; ++p) t = fma(D[i * kTrsmTPitchX + p], x[p], t);
            x[i] = i == lane ? T(1) : (i < lane ? T(0) : -t);
        }
        __syncwarp();
#pragma unroll
        for (int i = 0; i < 32; ++i) D[i * kTrsmTPitchX + lane] = x[i];
    }
    __syncthreads();
    for (int b = 0; b < nb; ++b) {
        const int rb = 32 * b, below = w - rb - 32;
        for (int i = warp; i < below; i += NW)
            trsm_copy_async(&Ls[i * kTrsmTPitchL + lane],
                            &A[(int64_t)(r + rb + 32 + i) * lda + r + rb + lane], true);
        {
            const T *D = Li + b * 32 * kTrsmTPitchX;
            T y[4] = {T(0), T(0), T(0), T(0)};
#pragma unroll 8
            for (int p = 0; p < 32; ++p) {
                const T xp = X[(rb + p) * kTrsmTPitchX + lane];
#pragma unroll
                for (int q = 0; q < 4; ++q) y[q] = fma(D[(4 * warp + q) * kTrsmTPitchX + p], xp, y[q]);
            }
            __syncthreads();
#pragma unroll
            for (int q = 0; q < 4; ++q) X[(rb + 4 * warp + q) * kTrsmTPitchX + lane] = y[q];
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        __syncthreads();
        if (below > 0) {
            T xb[32];
#pragma unroll
            for (int p = 0; p < 32; ++p) xb[p] = X[(rb + p) * kTrsmTPitchX + lane];
            for (int i = warp; i < below; i += NW) {
                const T *lr = Ls + i * kTrsmTPitchL;
                T t = T(0);
#pragma unroll
                for (int q = 0; q < 32; ++q) t = fma(lr[q], xb[q], t);
                X[(rb + 32 + i) * kTrsmTPitchX + lane] -= t;
            }
        }
        __syncthreads();
    }
    if (cv)
        for (int i = warp; i < w; i += NW) B[(int64_t)(r + i) * ldb + col] = X[i * kTrsmTPitchX + lane];
}

// The row moves of LAPACK-style interchanges ipiv[c .. c+w) (w <= 32), as a
// list: one warp replays the swaps on the positions they touch (lane k
// tracks position c + k and, from step k on, possibly one more), then lists
// every tracked position whose row changed.
__global__ void ipiv_moves_kernel(const int32_t *ipiv, int c, int w, int *mlist) {
    const unsigned full = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    int pos0 = c + lane, row0 = c + lane, pos1 = -1, row1 = -1;
    const int mine = lane < w ? ipiv[c + lane] : 0;
    for (int j = 0; j < w; ++j) {
        const int cj = c + j, p = __shfl_sync(full, mine, j);
        int h = pos0 == cj ? row0 : (pos1 == cj ? row1 : -1);
        unsigned m = __ballot_sync(full, h >= 0);
        const int at_cj = m ? __shfl_sync(full, h, __ffs(m) - 1) : cj;
        h = pos0 == p ? row0 : (pos1 == p ? row1 : -1);
        m = __ballot_sync(full, h >= 0);
        const int at_p = m ? __shfl_sync(full, h, __ffs(m) - 1) : p;
        const bool tracked = __any_sync(full, pos0 == p || pos1 == p);
        if (pos0 == cj) row0 = at_p;
        else if (pos0 == p) row0 = at_cj;
        if (pos1 == cj) row1 = at_p;
        else if (pos1 == p) row1 = at_cj;
        if (!tracked && lane == j) {
            pos1 = p;
            row1 = at_cj;
        }
    }
    const bool mv0 = row0 != pos0, mv1 = pos1 >= 0 && row1 != pos1;
    const unsigned b0 = __ballot_sync(full, mv0), b1 = __ballot_sync(full, mv1);
    const unsigned lt = (1u << lane) - 1u;
    if (mv0) {
        const int i = __popc(b0 & lt);
        mlist[1 + 2 * i] = row0;
        mlist[2 + 2 * i] = pos0;
    }
    if (mv1) {
        const int i = __popc(b0) + __popc(b1 & lt);
        mlist[1 + 2 * i] = row1;
        mlist[2 + 2 * i] = pos1;
    }
    if (lane == 0) mlist[0] = __popc(b0) + __popc(b1);
}

}  // namespace nmx
