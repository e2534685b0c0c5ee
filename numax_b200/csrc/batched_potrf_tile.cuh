// Batched Cholesky + cho_solve on 8 x 8 DMMA tiles (FP64), a second CTA
// shape for the plan of batched_potrf.cu: the same work as
// potrf_potrs_batched_kernel (numax's Array-tier cholesky + cholesky_solve,
// numax/linalg/_array/cholesky.mojo:26-92, per matrix of a ragged batch) in
// a layout built around mma.sync.m8n8k4.f64.
//
// A matrix's lower triangle is held in shared memory as 8 x 8 tiles, each
// stored row-major -- which is exactly the DMMA accumulator layout (lane l
// owns elements 2l and 2l + 1: row l/4, columns 2(l%4), 2(l%4) + 1) -- so
// every tile load and store is one conflict-free 16-byte access per lane.
// The right-hand sides ride as one more tile row: B^T (nrhs <= 8 rows) under
// the matrix, so the forward substitution y = L^-1 b is the panel solve of
// that row.  Per 8-column step K:
//   1. one warp factors the diagonal tile in registers (lane = an element
//      pair; the column's pivot, its scaling and the rank-1 update move by
//      shuffles) with numax's rule l_jj = sqrt(guard_nonzero(d, 1e-30)), and
//      forms W_K = L_KK^-1 in the same loop, off the pivot chain;
//   2. every tile (I, K) of the panel becomes L_IK = A_IK W_K^T: two DMMAs;
//      the result is stored as a tile and once more in A-fragment order
//      (element (m, k) of the k4 step q at [q][lane], lane = 4m + k % 4),
//      which is also the B-fragment order of L_IK^T;
//   3. the trailing tiles (I, J), K < J <= I, take A_IJ -= L_IK L_JK^T: two
//      DMMAs with both operands read in fragment order, conflict-free.
// The back substitution x = L^-T y runs as X^T = Y^T L^-1 over the stored
// tiles: for J from the last block up, the warps split the products
// X^T_I L_IJ (I > J) and one warp applies W_J.
#pragma once

namespace nmx {

constexpr int kTileNW = 8;  // warps per CTA of the tile kernel

// Shared-memory doubles for matrices with T = ceil(nmax / 8) tile rows:
// the tile store (lower tiles and the right-hand-side row), the panel in
// fragment order (reused for X^T in fragment order by the back solve), the
// diagonal tiles' inverses W_K and the back solve's per-warp partials.
__host__ __device__ inline int tile_smem_doubles(int nmax) {
    const int T = (nmax + 7) / 8;
    return (T * (T + 1) / 2 + T) * 64 + (T + 1) * 64 + T * 64 + kTileNW * 64;
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

template <int TMAX>
__device__ void potrf_tile_one(const BatchedPotrfArgs &args, int idx, double *smem) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int n = args.ns[idx], nrhs = args.nrhs;
    const int T = (n + 7) >> 3;
    const double *A = static_cast<const double *>(args.A) + args.a_off[idx];
    double *L = static_cast<double *>(args.L) + args.a_off[idx];
    const double *B = static_cast<const double *>(args.B) + args.b_off[idx];
    double *X = static_cast<double *>(args.X) + args.b_off[idx];
    const int tri_T = T * (T + 1) / 2;
    double *TS = smem;                       // (tri_T + T) tiles
    double *PB = TS + (tri_T + T) * 64;      // (T + 1) tiles, fragment order
    double *WS = PB + (T + 1) * 64;          // T tiles, row-major
    double *RED = WS + T * 64;               // kTileNW tiles
    auto slot = [&](int I, int J) { return I < T ? I * (I + 1) / 2 + J : tri_T + J; };

    // ---- load: lower tiles of A, and B^T as the last tile row ------------
    // Element e of the store: tile s = e / 64, (r, c) = ((e % 64) / 8, e % 8).
    // All copies in flight at once (cp.async); out of range (past n, or above
    // the diagonal) is zero-filled, and the padded diagonal entries then set
    // to 1 so that the padding factors to the identity.
    const int nel = (tri_T + T) * 64;
    const unsigned ts0 = (unsigned)__cvta_generic_to_shared(TS);
#pragma unroll 4
    for (int e = threadIdx.x; e < nel; e += kTileNW * 32) {
        const int s = e >> 6, r = (e >> 3) & 7, c = e & 7;
        const double *src = A;
        bool ok;
        if (s < tri_T) {
            int I = (int)((sqrtf(8.f * (float)s + 1.f) - 1.f) * 0.5f);
            I -= (I * (I + 1)) / 2 > s;
            I += ((I + 1) * (I + 2)) / 2 <= s;
            const int J = s - (I * (I + 1)) / 2;
            const int gi = 8 * I + r, gj = 8 * J + c;
            ok = gi < n && gj <= gi;
            if (ok) src = A + (int64_t)gi * n + gj;
        } else {
            const int gj = 8 * (s - tri_T) + c;
            ok = r < nrhs && gj < n;
            if (ok) src = B + (int64_t)gj * nrhs + r;
        }
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(ts0 + 8u * (unsigned)e),
                     "l"(src), "r"(ok ? 8 : 0)
                     : "memory");
    }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
    __syncthreads();
    if (threadIdx.x < 8 * T - n) {
        const int g = n + threadIdx.x, o = g - 8 * (T - 1);
        TS[slot(T - 1, T - 1) * 64 + 9 * o] = 1.0;
    }
    int info_local = 0;
    __syncthreads();

    for (int K = 0; K < T; ++K) {
        // ---- 1. diagonal tile (warp 0) -------------------------------------
        if (warp == 0) {
            double *tile = TS + slot(K, K) * 64;
            const double2 t = *reinterpret_cast<const double2 *>(tile + 2 * lane);
            double v0 = t.x, v1 = t.y;
            const int r = lane >> 2, c0 = 2 * (lane & 3);
            double w0 = (r == c0) ? 1.0 : 0.0, w1 = (r == c0 + 1) ? 1.0 : 0.0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const int src = 4 * j + (j >> 1);
                const double d = __shfl_sync(0xffffffffu, (j & 1) ? v1 : v0, src);
                if (lane == 0 && info_local == 0 && 8 * K + j < n && d <= 0.0)
                    info_local = 8 * K + j + 1;
                const double g = guard_nonzero(d, 1e-30);
                const double inv = rsqrt(g);
                const double ljj = g * inv;
                // Column j of L: the diagonal entry and the rows below scaled.
                if (c0 == j) v0 = (r == j) ? ljj : (r > j ? v0 * inv : v0);
                if (c0 + 1 == j) v1 = (r == j) ? ljj : (r > j ? v1 * inv : v1);
                const double col = (j & 1) ? v1 : v0;
                const double lrj = __shfl_sync(0xffffffffu, col, 4 * r + (j >> 1));
                const double lc0 = __shfl_sync(0xffffffffu, col, 4 * c0 + (j >> 1));
                const double lc1 = __shfl_sync(0xffffffffu, col, 4 * (c0 + 1) + (j >> 1));
                if (r > j) {
                    if (c0 > j && c0 <= r) v0 -= lrj * lc0;
                    if (c0 + 1 > j && c0 + 1 <= r) v1 -= lrj * lc1;
                }
                // W = L^-1 by forward elimination: row j is final once scaled,
                // then the rows below lose l_rj times it.
                if (r == j) {
                    w0 *= inv;
                    w1 *= inv;
                }
                const double wj0 = __shfl_sync(0xffffffffu, w0, 4 * j + (lane & 3));
                const double wj1 = __shfl_sync(0xffffffffu, w1, 4 * j + (lane & 3));
                if (r > j) {
                    w0 -= lrj * wj0;
                    w1 -= lrj * wj1;
                }
            }
            *reinterpret_cast<double2 *>(tile + 2 * lane) = make_double2(v0, v1);
            *reinterpret_cast<double2 *>(WS + K * 64 + 2 * lane) = make_double2(w0, w1);
            // L's diagonal tile: the lower triangle inside the matrix.
            const int gi = 8 * K + r, gj = 8 * K + c0;
            if (gi < n) {
                if (gj <= gi) L[(int64_t)gi * n + gj] = v0;
                if (gj + 1 <= gi) L[(int64_t)gi * n + gj + 1] = v1;
            }
        }
        __syncthreads();
        // ---- 2. panel: L_IK = A_IK W_K^T, I = K+1 .. T (T: the RHS row) ---
        {
            // B-fragments of W_K^T: element (k = 4q + l%4, n = l/4) = W[l/4][4q + l%4].
            const double b0 = WS[K * 64 + 8 * (lane >> 2) + (lane & 3)];
            const double b1 = WS[K * 64 + 8 * (lane >> 2) + 4 + (lane & 3)];
            for (int I = K + 1 + warp; I <= T; I += kTileNW) {
                double *tile = TS + slot(I, K) * 64;
                const double2 t = *reinterpret_cast<const double2 *>(tile + 2 * lane);
                const double a0 = afrag_of(t.x, t.y, 0, lane), a1 = afrag_of(t.x, t.y, 1, lane);
                double acc[2] = {0.0, 0.0};
                dmma8(acc, a0, b0);
                dmma8(acc, a1, b1);
                *reinterpret_cast<double2 *>(tile + 2 * lane) = make_double2(acc[0], acc[1]);
                PB[I * 64 + lane] = afrag_of(acc[0], acc[1], 0, lane);
                PB[I * 64 + 32 + lane] = afrag_of(acc[0], acc[1], 1, lane);
                if (I < T) {
                    const int gi = 8 * I + (lane >> 2), gj = 8 * K + 2 * (lane & 3);
                    if (gi < n) {
                        if (gj < n) L[(int64_t)gi * n + gj] = acc[0];
                        if (gj + 1 < n) L[(int64_t)gi * n + gj + 1] = acc[1];
                    }
                }
            }
        }
        __syncthreads();
        // ---- 3. trailing update: (I, J), K < J <= I <= T ---------------------
        {
            int q = 0;
            for (int J = K + 1; J < T; ++J) {
                const double bj0 = PB[J * 64 + lane], bj1 = PB[J * 64 + 32 + lane];
                for (int I = J; I <= T; ++I, ++q) {
                    if ((q % kTileNW) != warp) continue;
                    double *tile = TS + slot(I, J) * 64;
                    const double2 t = *reinterpret_cast<const double2 *>(tile + 2 * lane);
                    double acc[2] = {t.x, t.y};
                    dmma8(acc, -PB[I * 64 + lane], bj0);
                    dmma8(acc, -PB[I * 64 + 32 + lane], bj1);
                    *reinterpret_cast<double2 *>(tile + 2 * lane) = make_double2(acc[0], acc[1]);
                }
            }
        }
        __syncthreads();
    }
    if (warp == 0 && lane == 0) args.info[idx] = info_local;

    // ---- back substitution: X^T_J = (Y^T_J - sum_{I>J} X^T_I L_IJ) W_J --------
    if (nrhs > 0) {
        double *XA = PB;  // X^T_I in A-fragment order
        for (int J = T - 1; J >= 0; --J) {
            // Each warp's share of the products, I = J+1+warp, J+1+warp+8, ...
            double part[2] = {0.0, 0.0};
            for (int I = J + 1 + warp; I < T; I += kTileNW) {
                const double *lt = TS + slot(I, J) * 64;
                // B-fragment of L_IJ: element (k = 4q + l%4, n = l/4).
                const double b0 = lt[8 * (lane & 3) + (lane >> 2)];
                const double b1 = lt[8 * (4 + (lane & 3)) + (lane >> 2)];
                dmma8(part, XA[I * 64 + lane], b0);
                dmma8(part, XA[I * 64 + 32 + lane], b1);
            }
            *reinterpret_cast<double2 *>(RED + warp * 64 + 2 * lane) = make_double2(part[0], part[1]);
            __syncthreads();
            if (warp == 0) {
                const double2 y = *reinterpret_cast<const double2 *>(TS + slot(T, J) * 64 + 2 * lane);
                double s0 = y.x, s1 = y.y;
#pragma unroll
                for (int w = 0; w < kTileNW; ++w) {
                    const double2 p = *reinterpret_cast<const double2 *>(RED + w * 64 + 2 * lane);
                    s0 -= p.x;
                    s1 -= p.y;
                }
                // X^T_J = S W_J: B-fragment of W_J, element (k = 4q + l%4, n = l/4).
                const double *wt = WS + J * 64;
                const double b0 = wt[8 * (lane & 3) + (lane >> 2)];
                const double b1 = wt[8 * (4 + (lane & 3)) + (lane >> 2)];
                double x[2] = {0.0, 0.0};
                dmma8(x, afrag_of(s0, s1, 0, lane), b0);
                dmma8(x, afrag_of(s0, s1, 1, lane), b1);
                XA[J * 64 + lane] = afrag_of(x[0], x[1], 0, lane);
                XA[J * 64 + 32 + lane] = afrag_of(x[0], x[1], 1, lane);
                // X (n x nrhs row-major): X^T element (rhs l/4, row 8J + 2(l%4) + e).
                const int rr = lane >> 2, gj = 8 * J + 2 * (lane & 3);
                if (rr < nrhs) {
                    if (gj < n) X[(int64_t)gj * nrhs + rr] = x[0];
                    if (gj + 1 < n) X[(int64_t)(gj + 1) * nrhs + rr] = x[1];
                }
            }
            __syncthreads();
        }
    }
}

template <int TMAX>
__global__ void __launch_bounds__(kTileNW * 32, 4)
    potrf_tile_batched_kernel(BatchedPotrfArgs args, int begin, int end, int nmax, int *counter) {
    double *S = reinterpret_cast<double *>(bp_smem);
    __shared__ int s_item;
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
        __syncthreads();
        const int item = begin + s_item;
        __syncthreads();
        if (item >= end) break;
        potrf_tile_one<TMAX>(args, args.order[item], S);
        __syncthreads();
    }
}

}  // namespace nmx
