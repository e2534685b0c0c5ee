// Batched Cholesky + cho_solve on 8 x 8 DMMA tiles (computed in FP64; FP32
// batches are widened on load and rounded on store), the second kernel
// family of the plan in batched_potrf.cu: the same work as
// potrf_potrs_batched_kernel (numax's Array-tier cholesky + cholesky_solve,
// numax/linalg/_array/cholesky.mojo:26-92, per matrix of a ragged batch) in
// a layout built around mma.sync.m8n8k4.f64, for a group of WPM warps per
// matrix (one CTA = one group; several CTAs share an SM).
//
// Shared memory of a CTA: the lower triangle as 8 x 8 tiles (tile (I, J),
// J <= I, at slot I(I+1)/2 + J), the right-hand sides as the nrhs rows of B^T
// (block J: nrhs x 8, row-major) and the inverted pivots 1/l_jj.  Inside a
// tile, element (r, c) sits at 8r + 2((c/2) ^ g(r)) + c%2 with
// g(r) = 2((r/2)%2): the column pairs of rows 2, 3, 6, 7 swapped in halves.
// With that swizzle the three ways a tile is read are all conflict-free
// shared accesses, with no shuffles and no second copy:
//   accumulator (lane l: row l/4, columns 2(l%4), 2(l%4)+1, one double2),
//   A fragment, and B fragment of the transpose (lane l: row l/4, column
//   4q + l%4),
//   B fragment (lane l: row 4q + l%4, column l/4).
// A factored diagonal tile holds L_KK in its lower triangle and the strict
// lower triangle of W_K = L_KK^-1, transposed, in its upper triangle (the
// diagonal of W_K is the inverted pivots), so the panel and the back
// substitution read W_K without recomputing it.
//
// Per 8-column step K (two barriers):
//   1. panel: L_IK = A_IK W_K^T for every tile below the diagonal (two
//      tiles in flight per warp), and the right-hand sides' block
//      Y_K = B_K W_K^T (the forward substitution);
//   2. trailing update A_IJ -= L_IK L_JK^T, K < J <= I, and B_J -= Y_K L_JK^T.
//      One warp (rotating with K) takes tile (K+1, K+1) first and factors
//      it right away (the look-ahead: each lane a scalar 8 x 8 Cholesky of
//      its own copy, then W one column per lane), then a smaller share of the
//      remaining tiles; the other warps split the rest into contiguous runs,
//      two tiles in flight at a time.
// The back substitution X^T = Y^T L^-1 runs right-looking from the last
// block: X^T_J = S_J W_J (as X_J = W_J^T S_J^T, so both operands come from
// shared memory in fragment order), then S_I -= X^T_J L_JI for every I < J,
// spread over the warps.
#pragma once

namespace nmx {

// CTA shapes of the tile kernel in a plan's schedule: 1000 + threads.
constexpr int kTileShapeBase = 1000;
// Diagonal-tile factorization, in trailing-tile units, kept off its warp's share.
constexpr int kTileDiagUnits = 20;

__host__ __device__ inline bool is_tile_shape(int shape) {
    return shape == kTileShapeBase + 32 || shape == kTileShapeBase + 64 ||
           shape == kTileShapeBase + 128 || shape == kTileShapeBase + 256;
}

// Shared-memory doubles for matrices up to nmax with nrhs right-hand sides.
__host__ __device__ inline int tile_smem_doubles(int nmax, int nrhs) {
    const int T = (nmax + 7) / 8;
    return T * (T + 1) / 2 * 64 + T * 8 * nrhs + T * 8;
}

__device__ __forceinline__ int swz(int r, int c) {
    return 8 * r + 2 * ((c >> 1) ^ (((r >> 1) & 1) << 1)) + (c & 1);
}

__device__ __forceinline__ void dmma8(double (&c)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
        : "+d"(c[0]), "+d"(c[1])
        : "d"(a), "d"(b));
}

// A-fragment (k4 step q) of the tile whose accumulator pair (v0, v1) this
// lane holds: element (row l/4, column 4q + l%4), owned by lane
// 4(l/4) + 2q + (l%4)/2 as its element (l%4) & 1.
__device__ __forceinline__ double afrag_of(double v0, double v1, int q, int lane) {
    const int src = 4 * (lane >> 2) + 2 * q + ((lane & 3) >> 1);
    const double x0 = __shfl_sync(0xffffffffu, v0, src);
    const double x1 = __shfl_sync(0xffffffffu, v1, src);
    return (lane & 1) ? x1 : x0;
}

// Factors, in one warp, the diagonal tile K held (updated) in shared memory.
// Every lane runs the same scalar 8 x 8 Cholesky on its own register copy of
// the lower triangle (broadcast reads), so the pivot chain is rsqrt and two
// FMAs per column with no shuffles (numax's rule
// l_jj = sqrt(guard_nonzero(d, 1e-30)) as l_jj = g / sqrt(g)).
// W = L^-1 runs one column per lane.  Stores L_KK (lower triangle of the
// tile, and global L), W's strict lower triangle transposed into the tile's
// upper triangle, and the inverted pivots.  Returns the 1-based column of
// the first pivot d <= 0 among the tile's valid columns, 0 if none.
template <typename TM>
__device__ __forceinline__ int factor_diag_tile(double *tile, double *dinv, TM *L, int n, int K,
                                                int lane) {
    double a[8][8];
#pragma unroll
    for (int i = 0; i < 8; ++i)
#pragma unroll
        for (int p = 0; 2 * p <= i; ++p) {
            const double2 v = *reinterpret_cast<const double2 *>(tile + swz(i, 2 * p));
            a[i][2 * p] = v.x;
            if (2 * p + 1 <= i) a[i][2 * p + 1] = v.y;
        }
    const int valid = n - 8 * K;
    int first = 0;
    double inv[8];
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        const double d = a[j][j];
        if (first == 0 && j < valid && d <= 0.0) first = j + 1;
        const double g = guard_nonzero(d, 1e-30);
        inv[j] = rsqrt(g);
        a[j][j] = g * inv[j];
#pragma unroll
        for (int i = j + 1; i < 8; ++i) a[i][j] *= inv[j];
#pragma unroll
        for (int i = j + 1; i < 8; ++i)
#pragma unroll
            for (int k = j + 1; k <= i; ++k) a[i][k] -= a[i][j] * a[k][j];
    }
    // Lane l: column c = l % 8 of W = L^-1 (lanes 8.. repeat it), with
    // w_j = 0 above the diagonal: w_i = (delta_ic - sum_{j<i} l_ij w_j) / l_ii.
    const int c = lane & 7;
    double w[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        double sum = (i == c) ? 1.0 : 0.0;
#pragma unroll
        for (int j = 0; j < i; ++j) sum -= a[i][j] * w[j];
        w[i] = sum * inv[i];
    }
    __syncwarp();
    // L's lower triangle (every lane stores the same values), W's strict
    // lower triangle transposed (lane c: position (c, i) = W[i][c], i > c),
    // the inverted pivots.
#pragma unroll
    for (int i = 0; i < 8; ++i) {
#pragma unroll
        for (int p = 0; 2 * p + 1 <= i; ++p)
            *reinterpret_cast<double2 *>(tile + swz(i, 2 * p)) = make_double2(a[i][2 * p], a[i][2 * p + 1]);
        if ((i & 1) == 0) tile[swz(i, i)] = a[i][i];
    }
    if (lane < 8) {
#pragma unroll
        for (int i = 1; i < 8; ++i)
            if (i > c) tile[swz(c, i)] = w[i];
    }
#pragma unroll
    for (int p = 0; p < 4; ++p)
        *reinterpret_cast<double2 *>(dinv + 8 * K + 2 * p) = make_double2(inv[2 * p], inv[2 * p + 1]);
    __syncwarp();
    const int r = lane >> 2, c0 = 2 * (lane & 3);
    const double2 v = *reinterpret_cast<const double2 *>(tile + swz(r, c0));
    const int gi = 8 * K + r, gj = 8 * K + c0;
    if (gi < n) {
        if (gj <= gi) L[(int64_t)gi * n + gj] = (TM)v.x;
        if (gj + 1 <= gi) L[(int64_t)gi * n + gj + 1] = (TM)v.y;
    }
    return first;
}

// Row gi, columns gj and gj + 1 (gj even) of an n-column row-major matrix
// of TM (double, or float rounded from the FP64 values).
template <typename TM>
__device__ __forceinline__ void store_pair(TM *M, int n, int gi, int gj, double x0, double x1) {
    if (gi >= n) return;
    TM *p = M + (int64_t)gi * n + gj;
    if (gj + 1 < n && (reinterpret_cast<uintptr_t>(p) & (2 * sizeof(TM) - 1)) == 0) {
        if constexpr (sizeof(TM) == 8)
            *reinterpret_cast<double2 *>(p) = make_double2(x0, x1);
        else
            *reinterpret_cast<float2 *>(p) = make_float2((float)x0, (float)x1);
    } else {
        if (gj < n) p[0] = (TM)x0;
        if (gj + 1 < n) p[1] = (TM)x1;
    }
}

template <int WPM>
__device__ __forceinline__ void group_sync() {
    if (WPM == 1)
        __syncwarp();
    else
        __syncthreads();
}

// Roles rotate over the warps so that co-resident CTAs, and the steps of one
// matrix, spread the serial diagonal work over the SM's schedulers: tile D's
// diagonal factorization runs in warp (D + off) % WPM, right-hand-side block
// I of the back substitution in warp (I + off) % WPM, with `off` per CTA.
// TIO: the batch's element type.  FP32 batches are loaded into the same FP64
// tiles and computed in FP64; L and X are rounded to FP32 on the way out.
template <int WPM, typename TIO>
__device__ void potrf_tile_one(const BatchedPotrfArgs &args, int idx, double *smem, int off,
                               int *s_info) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int M = WPM - 1;  // WPM is a power of two
    const int n = args.ns[idx], nrhs = args.nrhs;
    const int T = (n + 7) >> 3;
    const TIO *A = static_cast<const TIO *>(args.A) + args.a_off[idx];
    TIO *L = static_cast<TIO *>(args.L) + args.a_off[idx];
    const TIO *B = static_cast<const TIO *>(args.B) + args.b_off[idx];
    TIO *X = static_cast<TIO *>(args.X) + args.b_off[idx];
    double *TS = smem;                        // T(T+1)/2 tiles, swizzled
    double *RB = TS + T * (T + 1) / 2 * 64;   // T blocks of nrhs x 8: B^T, Y^T, X^T
    double *DI = RB + T * 8 * nrhs;           // 8T inverted pivots
    const int r = lane >> 2, cp = lane & 3;   // accumulator row, column pair
    auto tile = [&](int I, int J) { return TS + (I * (I + 1) / 2 + J) * 64; };
    auto rb_afrag = [&](int J, int q) -> double {
        return r < nrhs ? RB[J * 8 * nrhs + r * 8 + 4 * q + cp] : 0.0;
    };

    // ---- load: the lower tiles of A and B^T, all copies in flight ----------
    // Warp w takes tiles w, w + WPM, ... in slot order; lane l the elements
    // (l/4, 2(l%4)) and (l/4, 2(l%4) + 1), as one 16-byte copy when the pair
    // is in range and aligned.  Out of range (past n, or above the diagonal)
    // is zero-filled.
    if constexpr (sizeof(TIO) == 8) {
        const unsigned ts0 = (unsigned)__cvta_generic_to_shared(TS);
        const int ntile = T * (T + 1) / 2;
        int I = 0, J = warp;
        while (J > I) {
            J -= I + 1;
            ++I;
        }
        for (int s = warp; s < ntile; s += WPM) {
            const int gi = 8 * I + r, gj = 8 * J + 2 * cp;
            const bool ok0 = gi < n && gj <= gi, ok1 = gi < n && gj + 1 <= gi;
            const double *src = ok0 ? A + (int64_t)gi * n + gj : A;
            const unsigned dst = ts0 + 8u * (unsigned)(s * 64 + swz(r, 2 * cp));
            if (ok1 && (reinterpret_cast<uintptr_t>(src) & 15) == 0) {
                asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(dst), "l"(src)
                             : "memory");
            } else {
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src),
                             "r"(ok0 ? 8 : 0)
                             : "memory");
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst + 8u),
                             "l"(ok1 ? src + 1 : A), "r"(ok1 ? 8 : 0)
                             : "memory");
            }
            J += WPM;
            while (J > I) {
                J -= I + 1;
                ++I;
            }
        }
        const unsigned rb0 = (unsigned)__cvta_generic_to_shared(RB);
        for (int e = threadIdx.x; e < T * 8 * nrhs; e += WPM * 32) {
            const int Jb = e / (8 * nrhs), rem = e - Jb * 8 * nrhs, rr = rem >> 3, cc = rem & 7;
            const int gj = 8 * Jb + cc;
            const bool ok = gj < n;
            const double *src = ok ? B + (int64_t)gj * nrhs + rr : B;
            asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(
                             rb0 + 8u * (unsigned)e),
                         "l"(src), "r"(ok ? 8 : 0)
                         : "memory");
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
    } else {
        // FP32: the elements go by cp.async (all in flight) to FP32 slots at
        // the start of the tile region, element e (tile slot * 64 + swizzled
        // position) at float index e; then they are widened in place from the
        // top down: element e's FP64 value overwrites only the FP32 slots of
        // elements 2e and 2e + 1, already read by then.
        float *TF = reinterpret_cast<float *>(TS);
        const unsigned tf0 = (unsigned)__cvta_generic_to_shared(TF);
        const int ntile = T * (T + 1) / 2;
        int I = 0, J = warp;
        while (J > I) {
            J -= I + 1;
            ++I;
        }
        for (int s = warp; s < ntile; s += WPM) {
            const int gi = 8 * I + r, gj = 8 * J + 2 * cp;
            const bool ok0 = gi < n && gj <= gi, ok1 = gi < n && gj + 1 <= gi;
            const TIO *src = ok0 ? A + (int64_t)gi * n + gj : A;
            const unsigned dst = tf0 + 4u * (unsigned)(s * 64 + swz(r, 2 * cp));
            if (ok1 && (reinterpret_cast<uintptr_t>(src) & 7) == 0) {
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(dst), "l"(src)
                             : "memory");
            } else {
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src),
                             "r"(ok0 ? 4 : 0)
                             : "memory");
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst + 4u),
                             "l"(ok1 ? src + 1 : A), "r"(ok1 ? 4 : 0)
                             : "memory");
            }
            J += WPM;
            while (J > I) {
                J -= I + 1;
                ++I;
            }
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
        group_sync<WPM>();
        constexpr int kPer = 8;  // elements per thread per chunk
        constexpr int kChunk = kPer * WPM * 32;
        const int nel = ntile * 64;
        for (int top = nel; top > 0; top -= kChunk) {
            const int lo = max(0, top - kChunk);
            float v[kPer];
#pragma unroll
            for (int u = 0; u < kPer; ++u) {
                const int e = lo + threadIdx.x + u * WPM * 32;
                v[u] = e < top ? TF[e] : 0.f;
            }
            group_sync<WPM>();
#pragma unroll
            for (int u = 0; u < kPer; ++u) {
                const int e = lo + threadIdx.x + u * WPM * 32;
                if (e < top) TS[e] = (double)v[u];
            }
            group_sync<WPM>();
        }
        for (int e = threadIdx.x; e < T * 8 * nrhs; e += WPM * 32) {
            const int Jb = e / (8 * nrhs), rem = e - Jb * 8 * nrhs, rr = rem >> 3, cc = rem & 7;
            const int gj = 8 * Jb + cc;
            RB[e] = gj < n ? (double)B[(int64_t)gj * nrhs + rr] : 0.0;
        }
    }
    group_sync<WPM>();
    if (warp == (off & M)) {
        // The padded diagonal entries (at most 7) set to 1 so that the
        // padding factors to the identity; then the first diagonal tile.
        if (lane < 8 * T - n) {
            const int o = n + lane - 8 * (T - 1);
            tile(T - 1, T - 1)[swz(o, o)] = 1.0;
        }
        __syncwarp();
        const int bad = factor_diag_tile(tile(0, 0), DI, L, n, 0, lane);
        if (lane == 0) *s_info = bad;
    }
    group_sync<WPM>();

    for (int K = 0; K < T; ++K) {
        // ---- 1. panel: L_IK = A_IK W_K^T (I = K+1 .. T-1), Y_K = B_K W_K^T ----
        {
            // B-fragment of W_K^T: element (k = 4q + l%4, col l/4) = W[l/4][k]:
            // below the diagonal in the tile's upper triangle, on it the
            // inverted pivot, above it zero.
            const double *tk = tile(K, K);
            double b[2];
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int k = 4 * q + cp;
                const double t = tk[swz(k, r)];
                b[q] = k < r ? t : (k == r ? DI[8 * K + r] : 0.0);
            }
            const int prank = (warp - off) & M;
            for (int I = K + 1 + prank; I < T; I += 2 * WPM) {
                // Two tiles in flight: both read before either is stored.
                const bool has_b = I + WPM < T;
                double *ta = tile(I, K), *tb = tile(has_b ? I + WPM : I, K);
                const double a0 = ta[swz(r, cp)], a1 = ta[swz(r, 4 + cp)];
                const double e0 = tb[swz(r, cp)], e1 = tb[swz(r, 4 + cp)];
                double xa[2] = {0.0, 0.0}, xb[2] = {0.0, 0.0};
                dmma8(xa, a0, b[0]);
                dmma8(xb, e0, b[0]);
                dmma8(xa, a1, b[1]);
                dmma8(xb, e1, b[1]);
                *reinterpret_cast<double2 *>(ta + swz(r, 2 * cp)) = make_double2(xa[0], xa[1]);
                store_pair(L, n, 8 * I + r, 8 * K + 2 * cp, xa[0], xa[1]);
                if (has_b) {
                    *reinterpret_cast<double2 *>(tb + swz(r, 2 * cp)) = make_double2(xb[0], xb[1]);
                    store_pair(L, n, 8 * (I + WPM) + r, 8 * K + 2 * cp, xb[0], xb[1]);
                }
            }
            if (nrhs > 0 && prank == ((T - 1 - K) & M)) {
                double acc[2] = {0.0, 0.0};
                dmma8(acc, rb_afrag(K, 0), b[0]);
                dmma8(acc, rb_afrag(K, 1), b[1]);
                if (r < nrhs)
                    *reinterpret_cast<double2 *>(RB + K * 8 * nrhs + r * 8 + 2 * cp) =
                        make_double2(acc[0], acc[1]);
            }
        }
        group_sync<WPM>();
        // ---- 2. trailing update --------------------------------------------
        // Units: tiles (I, J), K < J <= I < T, in order J ascending, I from J;
        // unit 0 is (K+1, K+1).
        const int nt = T - K - 1;
        if (nt > 0) {
            const int U = nt * (nt + 1) / 2;
            // Rank 0 is the warp that factors tile (K+1, K+1).
            const int rank = (warp - (K + 1 + off)) & M;
            int u0, u1;  // this warp's run of units 1 .. U-1
            if (WPM == 1) {
                u0 = 1;
                u1 = U;
            } else {
                const int c0 = max(0, (U - 1 - kTileDiagUnits * (WPM - 1)) / WPM);
                constexpr int others = WPM > 1 ? WPM - 1 : 1;
                const int per = (U - 1 - c0 + others - 1) / others;
                if (rank == 0) {
                    u0 = 1;
                    u1 = 1 + c0;
                } else {
                    u0 = min(U, 1 + c0 + (rank - 1) * per);
                    u1 = min(U, u0 + per);
                }
            }
            if (rank == 0) {
                // Tile (K+1, K+1) updated first, then factored.
                const int D = K + 1;
                const double *td = tile(D, K);
                double *tc = tile(D, D);
                const double2 v = *reinterpret_cast<const double2 *>(tc + swz(r, 2 * cp));
                double acc[2] = {v.x, v.y};
                dmma8(acc, -td[swz(r, cp)], td[swz(r, cp)]);
                dmma8(acc, -td[swz(r, 4 + cp)], td[swz(r, 4 + cp)]);
                *reinterpret_cast<double2 *>(tc + swz(r, 2 * cp)) = make_double2(acc[0], acc[1]);
                __syncwarp();
                const int bad = factor_diag_tile(tc, DI, L, n, D, lane);
                if (lane == 0 && bad && *s_info == 0) *s_info = 8 * D + bad;
            }
            if (u0 < u1) {
                int J = K + 1, I = u0;
                while (I >= T - J) {
                    I -= T - J;
                    ++J;
                }
                I += J;
                for (int u = u0; u < u1; u += 2) {
                    // Two units in flight: all operands read before either store.
                    const int Ja = J, Ia = I;
                    if (++I == T) I = ++J;
                    const bool has_b = u + 1 < u1;
                    const int Jb = has_b ? J : Ja, Ib = has_b ? I : Ia;
                    if (has_b && ++I == T) I = ++J;
                    const double *pa = tile(Ia, K), *qa = tile(Ja, K);
                    const double *pb = tile(Ib, K), *qb = tile(Jb, K);
                    double *ca = tile(Ia, Ja), *cb = tile(Ib, Jb);
                    const double a0 = pa[swz(r, cp)], a1 = pa[swz(r, 4 + cp)];
                    const double ba0 = qa[swz(r, cp)], ba1 = qa[swz(r, 4 + cp)];
                    const double e0 = pb[swz(r, cp)], e1 = pb[swz(r, 4 + cp)];
                    const double bb0 = qb[swz(r, cp)], bb1 = qb[swz(r, 4 + cp)];
                    const double2 va = *reinterpret_cast<const double2 *>(ca + swz(r, 2 * cp));
                    const double2 vb = *reinterpret_cast<const double2 *>(cb + swz(r, 2 * cp));
                    double xa[2] = {va.x, va.y}, xb[2] = {vb.x, vb.y};
                    dmma8(xa, -a0, ba0);
                    dmma8(xb, -e0, bb0);
                    dmma8(xa, -a1, ba1);
                    dmma8(xb, -e1, bb1);
                    *reinterpret_cast<double2 *>(ca + swz(r, 2 * cp)) = make_double2(xa[0], xa[1]);
                    if (has_b)
                        *reinterpret_cast<double2 *>(cb + swz(r, 2 * cp)) = make_double2(xb[0], xb[1]);
                }
            }
            // Right-hand sides: B_J -= Y_K L_JK^T, J = K+1 .. T-1, from the last rank down.
            if (nrhs > 0) {
                const double y0 = rb_afrag(K, 0), y1 = rb_afrag(K, 1);
                for (int J = K + 1 + (M - rank); J < T; J += WPM) {
                    const double *q = tile(J, K);
                    double *yc = RB + J * 8 * nrhs + r * 8 + 2 * cp;
                    double acc[2] = {0.0, 0.0};
                    if (r < nrhs) {
                        acc[0] = yc[0];
                        acc[1] = yc[1];
                    }
                    dmma8(acc, -y0, q[swz(r, cp)]);
                    dmma8(acc, -y1, q[swz(r, 4 + cp)]);
                    if (r < nrhs) *reinterpret_cast<double2 *>(yc) = make_double2(acc[0], acc[1]);
                }
            }
        }
        group_sync<WPM>();
    }
    if (threadIdx.x == 0) args.info[idx] = *s_info;

    // ---- back substitution, right-looking: X^T_J = S_J W_J once every block
    // below has been applied, then S_I -= X^T_J L_JI for I < J.  Block I's S
    // lives in RB and is only touched by its owner warp, which finishes block
    // J-1 right after applying X_J to it; one barrier per block.
    if (nrhs > 0) {
        auto finish_block = [&](int J) {
            // X_J = W_J^T S_J^T (8 x nrhs): A = W_J^T, element (m = l/4,
            // k = 4q + l%4) = W[k][m], below W's diagonal at the tile's
            // transposed position (m, k); B = S_J^T, element (k, rhs l/4),
            // read from RB row-major.  No shuffles.
            __syncwarp();
            const double *tj = tile(J, J);
            double *yj = RB + J * 8 * nrhs;
            double x[2] = {0.0, 0.0};
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int k = 4 * q + cp;
                const double t = tj[swz(r, k)];
                const double wa = k > r ? t : (k == r ? DI[8 * J + r] : 0.0);
                dmma8(x, wa, rb_afrag(J, q));
            }
            __syncwarp();
            // Lane (row r, rhs 2cp and 2cp + 1): X^T back into RB, X to global.
            const int gj = 8 * J + r;
#pragma unroll
            for (int e = 0; e < 2; ++e) {
                const int h = 2 * cp + e;
                if (h < nrhs) {
                    yj[h * 8 + r] = x[e];
                    if (gj < n) X[(int64_t)gj * nrhs + h] = (TIO)x[e];
                }
            }
        };
        if (warp == ((T - 1 + off) & M)) finish_block(T - 1);
        group_sync<WPM>();
        for (int J = T - 1; J > 0; --J) {
            const double x0 = -rb_afrag(J, 0), x1 = -rb_afrag(J, 1);
            // Largest I <= J-1 owned by this warp, then down by WPM.
            for (int I = J - 1 - ((J - 1 + off - warp) & M); I >= 0; I -= WPM) {
                const double *t = tile(J, I);
                double *yi = RB + I * 8 * nrhs + r * 8 + 2 * cp;
                double acc[2] = {0.0, 0.0};
                if (r < nrhs) {
                    acc[0] = yi[0];
                    acc[1] = yi[1];
                }
                // B-fragment of L_JI: element (k = 4q + l%4, col l/4).
                dmma8(acc, x0, t[swz(cp, r)]);
                dmma8(acc, x1, t[swz(4 + cp, r)]);
                if (r < nrhs) *reinterpret_cast<double2 *>(yi) = make_double2(acc[0], acc[1]);
                if (I == J - 1) finish_block(J - 1);
            }
            group_sync<WPM>();
        }
    }
}

// Registers capped so that the shapes meant for small matrices keep many
// CTAs per SM: 16 one-warp, 8 two-warp, 3 four-warp, 2 eight-warp CTAs.
template <int WPM, typename TIO>
__global__ void __launch_bounds__(WPM * 32, WPM == 4 ? 3 : 512 / (WPM * 32))
    potrf_tile_batched_kernel(BatchedPotrfArgs args, int begin, int end, int nmax, int *counter) {
    double *S = reinterpret_cast<double *>(bp_smem);
    __shared__ int s_item, s_off, s_info;
    if (threadIdx.x == 0) {
        // This CTA's warp slots on the SM (a hint only): co-resident CTAs
        // start their role rotation at different warps.
        unsigned wid;
        asm volatile("mov.u32 %0, %%warpid;" : "=r"(wid));
        s_off = (int)(wid / WPM);
    }
    for (;;) {
        if (threadIdx.x == 0) {
            s_item = atomicAdd(counter, 1);
            s_info = 0;
        }
        __syncthreads();
        const int item = begin + s_item, off = s_off;
        __syncthreads();
        if (item >= end) break;
        potrf_tile_one<WPM, TIO>(args, args.order[item], S, off, &s_info);
        __syncthreads();
    }
}

}  // namespace nmx
