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
// reduces, in one vector, the dot products of the new reflector with the
// remaining panel columns and the pieces of the next column's norm (every
// CTA sums the same partials in the same order, so all agree on beta and
// tau); the norm is downdated from them, with an exact recompute when
// cancellation would cost accuracy.  The same pass accumulates the panel's
// Gram matrix V^T V for T and writes V densely (unit diagonal, zeros above)
// for the GEMMs.  numax's reflector convention is kept exactly:
// beta = -sign(alpha) ||x|| (alpha <= 0 gives +||x||), tau = (beta-alpha)/beta,
// v = x / (alpha - beta), tau = 0 when the sub-column is exactly zero.
#include <algorithm>

#include "dense_common.cuh"

namespace nmx {

constexpr int kQrW = 16;  // panel width (numax's default block)
constexpr int kQrThreads = 512;

// Per-CTA partial vector of one reduction round of the panel: [0, 16) the
// dot products v^T a_c with the panel's remaining columns, then the pieces of
// the next column's norm below its diagonal (S_aa = sum a^2, S_av = sum v a,
// S_vv = sum v^2 over the rows below the next diagonal), and that column's
// diagonal entry and v there (from the CTA that owns the row).
// Then [21, 37): the Gram column of the new reflector, v_i^T v_j for i < j.
constexpr int kQrVec = 37;
constexpr int kQrSaa = 16, kQrSav = 17, kQrSvv = 18, kQrA1 = 19, kQrV1 = 20, kQrGram = 21;
constexpr int kQrSub = 12;    // sub-sums per element of the cross-CTA sum
constexpr int kQrMaxG = 192;  // most CTAs of the panel kernel
constexpr int kQrPart = kQrMaxG;  // partials stored element-major: [kQrVec][kQrMaxG]
// The next column's norm is downdated from the sums above (one grid barrier
// per column); it is recomputed exactly, with one more barrier, when the
// downdated value is below this fraction of the magnitude of its terms.
constexpr double kQrDowndateTol = 0.5;

template <typename T>
struct QrScratch {
    T *part;        // [2][kQrVec][kQrPart] per-CTA partials (double-buffered)
    T *gram_part;   // [kQrW * kQrW]: V^T V for larft_kernel
    unsigned *bar;
    int *err;
};

// T of the block reflector (w x w upper triangular) from the strict upper
// Gram entries g[p][i] = v_p^T v_i and the taus, numax's larft
// (numax/linalg/panel.mojo:2076-2169): t_ii = tau_i and
// t[q][i] = sum_{q<=r<i} t[q][r] (-tau_i g[r][i]), column by column, the rows
// q of a column in parallel.  One warp (lanes 0..w-1 do the rows).
template <typename T>
__device__ void build_t(const T (*g)[kQrW], const T *taus, int w, T (*t)[kQrW]) {
    const int q = threadIdx.x & 31;
    for (int e = q; e < kQrW * kQrW; e += 32) t[e / kQrW][e % kQrW] = T(0);
    __syncwarp();
    for (int i = 0; i < w; ++i) {
        if (q < i) t[q][i] = -taus[i] * g[q][i];
        __syncwarp();
        T sum = T(0);
        if (q < i)
            for (int r = q; r < i; ++r) sum += t[q][r] * t[r][i];
        __syncwarp();
        if (q < i) t[q][i] = sum;
        if (q == i) t[i][i] = taus[i];
        __syncwarp();
    }
}

// Tm = T or T^T (kQrW x kQrW, zero outside w x w), by one warp.
template <typename T>
__device__ void store_t(const T (*t)[kQrW], int transposed, T *Tm) {
    for (int e = threadIdx.x & 31; e < kQrW * kQrW; e += 32) {
        const int p = e / kQrW, q = e - p * kQrW;
        Tm[e] = transposed ? t[q][p] : t[p][q];
    }
}

// One reduction round: this CTA's partial vector p (per thread) is summed
// over the block and published, then after the grid barrier every CTA sums
// all CTAs' vectors in the same fixed order (so all agree bit for bit) into
// tot.  Returns false if the barrier gave up.
template <typename T>
__device__ __forceinline__ bool reduce_round(T (&p)[kQrVec], QrScratch<T> &sc, unsigned &gen,
                                             T *wred, T *sub, T *tot, int *s_flag) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, G = gridDim.x;
#pragma unroll
    for (int i = 0; i < kQrVec; ++i) {
        T v = p[i];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) wred[warp * kQrVec + i] = v;
    }
    __syncthreads();
    T *slot = sc.part + (size_t)(gen & 1) * kQrVec * kQrPart;
    if (threadIdx.x < kQrVec) {
        T t = T(0);
#pragma unroll
        for (int w = 0; w < kQrThreads / 32; ++w) t += wred[w * kQrVec + threadIdx.x];
        slot[(size_t)threadIdx.x * kQrPart + blockIdx.x] = t;
    }
    if (!grid_barrier(sc.bar, gen++, (unsigned)G, sc.err, s_flag)) return false;
    if (threadIdx.x < kQrVec * kQrSub) {
        // All of this thread's loads in flight at once, then summed in order.
        constexpr int kPer = (kQrMaxG + kQrSub - 1) / kQrSub;
        const int i = threadIdx.x / kQrSub, s = threadIdx.x - i * kQrSub;
        const T *src = slot + (size_t)i * kQrPart;
        T v[kPer];
#pragma unroll
        for (int u = 0; u < kPer; ++u) {
            const int g = s + u * kQrSub;
            v[u] = g < G ? __ldcg(src + g) : T(0);
        }
        T acc = T(0);
#pragma unroll
        for (int u = 0; u < kPer; ++u) acc += v[u];
        sub[i * kQrSub + s] = acc;
    }
    __syncthreads();
    if (threadIdx.x < kQrVec) {
        T acc = T(0);
#pragma unroll
        for (int q = 0; q < kQrSub; ++q) acc += sub[threadIdx.x * kQrSub + q];
        tot[threadIdx.x] = acc;
    }
    __syncthreads();
    return true;
}

// Factor panel columns [k, k+w) over rows [k, m) in place; Vd receives V
// (rows [k, m) x w, row-major ld kQrW) and tau[k..k+w) the scales.  One
// reduction round (one grid barrier) per column: the round after column j's
// reflector carries its dot products with the remaining panel columns and
// the pieces of column j+1's norm, which every CTA then downdates itself.
template <typename T>
__global__ void __launch_bounds__(kQrThreads, 1)
    geqr2_coop_kernel(T *A, int64_t lda, int m, int k, int w, int rows_per_cta, T *tau, T *Vd,
                      T *Tm, int transposed, QrScratch<T> sc) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int ldl = kQrW + 1;
    T *loc = reinterpret_cast<T *>(smem_raw);
    __shared__ T wred[(kQrThreads / 32) * kQrVec];
    __shared__ T sub[kQrVec * kQrSub];
    __shared__ T tot[kQrVec];
    __shared__ T s_gram[kQrW][kQrW], s_t[kQrW][kQrW], s_tau[kQrW], s_f[kQrW];
    __shared__ int s_flag;
    const int cta = blockIdx.x, tid = threadIdx.x;
    const int r0 = k + cta * rows_per_cta;
    const int nloc = max(0, min(rows_per_cta, m - r0));
    {
        // Every copy in flight at once.
        const unsigned l0 = (unsigned)__cvta_generic_to_shared(loc);
        for (int e = tid; e < nloc * w; e += kQrThreads) {
            const int r = e / w, j = e - r * w;
            const T *src = A + (int64_t)(r0 + r) * lda + k + j;
            if constexpr (sizeof(T) == 8)
                asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(
                                 l0 + (unsigned)(sizeof(T) * (r * ldl + j))),
                             "l"(src)
                             : "memory");
            else
                asm volatile("cp.async.ca.shared.global [%0], [%1], 4;\n" ::"r"(
                                 l0 + (unsigned)(sizeof(T) * (r * ldl + j))),
                             "l"(src)
                             : "memory");
        }
        asm volatile("cp.async.wait_all;\n" ::: "memory");
    }
    __syncthreads();
    unsigned gen = 0;
    // Column 0: its norm below the diagonal and its diagonal entry.
    T alpha, below;
    {
        T p[kQrVec];
#pragma unroll
        for (int i = 0; i < kQrVec; ++i) p[i] = T(0);
        for (int r = tid; r < nloc; r += kQrThreads) {
            const int gr = r0 + r;
            const T x = loc[r * ldl];
            if (gr > k) p[kQrSaa] += x * x;
            else if (gr == k) p[kQrA1] = x;
        }
        if (!reduce_round(p, sc, gen, wred, sub, tot, &s_flag)) return;
        alpha = tot[kQrA1];
        below = tot[kQrSaa];
    }
    for (int j = 0; j < w; ++j) {
        const int col = k + j;
        // numax's reflector: beta = -sign(alpha) ||x||, tau = (beta - alpha) / beta,
        // v = x / (alpha - beta); no reflection when the sub-column is zero.
        T this_tau = T(0), scale = T(0), beta = alpha;
        const bool reflect = below != T(0);
        if (reflect) {
            beta = sqrt(alpha * alpha + below);
            if (alpha > T(0)) beta = -beta;
            this_tau = (beta - alpha) / beta;
            scale = T(1) / (alpha - beta);
            for (int r = tid; r < nloc; r += kQrThreads) {
                const int gr = r0 + r;
                if (gr > col) loc[r * ldl + j] *= scale;
                else if (gr == col) loc[r * ldl + j] = beta;
            }
        }
        if (cta == 0 && tid == 0) tau[col] = this_tau;
        if (tid == 0) s_tau[j] = this_tau;
        const bool more = j + 1 < w;
        __syncthreads();
        // The round: v_j's Gram column; unless j is the panel's last column,
        // its dot products with the remaining columns and column j+1's norm
        // pieces.
        T p[kQrVec];
#pragma unroll
        for (int i = 0; i < kQrVec; ++i) p[i] = T(0);
        // Every column accumulates (no per-column tests); only the entries
        // the round needs are read afterwards: dots for j < c < w, Gram for c < j.
        for (int r = tid; r < nloc; r += kQrThreads) {
            const int gr = r0 + r;
            if (gr < col) continue;
            const T *row = loc + r * ldl;
            if (gr == col) {
#pragma unroll
                for (int c = 0; c < kQrW; ++c) {
                    const T x = row[c];
                    p[c] += x;
                    p[kQrGram + c] += x;
                }
            } else {
                const T v = row[j];
#pragma unroll
                for (int c = 0; c < kQrW; ++c) {
                    const T x = row[c];
                    p[c] += v * x;
                    p[kQrGram + c] += x * v;
                }
                if (more) {
                    const T a = row[j + 1];
                    if (gr == col + 1) {
                        p[kQrA1] = a;
                        p[kQrV1] = v;
                    } else {
                        p[kQrSaa] += a * a;
                        p[kQrSav] += v * a;
                        p[kQrSvv] += v * v;
                    }
                }
            }
        }
        if (!reduce_round(p, sc, gen, wred, sub, tot, &s_flag)) return;
        if (tid < j) s_gram[tid][j] = tot[kQrGram + tid];
        if (!more) break;
        if (tid < kQrW) s_f[tid] = (tid > j && tid < w) ? this_tau * tot[tid] : T(0);
        __syncthreads();
        // a_c -= (tau d_c) v for the remaining panel columns (v_col = 1; the
        // factor is zero past the panel's width).
        for (int r = tid; r < nloc; r += kQrThreads) {
            const int gr = r0 + r;
            if (gr < col) continue;
            T *row = loc + r * ldl;
            const T v = gr == col ? T(1) : row[j];
#pragma unroll
            for (int c = 0; c < kQrW; ++c)
                if (c > j) row[c] = fma(-s_f[c], v, row[c]);
        }
        // Column j+1: its diagonal entry after the update (the same fma the
        // owner applied) and its norm below the diagonal, downdated.
        const T f = this_tau * tot[j + 1];
        const T saa = tot[kQrSaa], sav = tot[kQrSav], svv = tot[kQrSvv];
        alpha = fma(-f, tot[kQrV1], tot[kQrA1]);
        T bl = saa - T(2) * f * sav + f * f * svv;
        if (!(bl >= T(kQrDowndateTol) * (saa + f * f * svv))) {
            __syncthreads();
            T q[kQrVec];
#pragma unroll
            for (int i = 0; i < kQrVec; ++i) q[i] = T(0);
            for (int r = tid; r < nloc; r += kQrThreads)
                if (r0 + r > col + 1) {
                    const T x = loc[r * ldl + j + 1];
                    q[kQrSaa] += x * x;
                }
            if (!reduce_round(q, sc, gen, wred, sub, tot, &s_flag)) return;
            bl = tot[kQrSaa];
        }
        below = bl;
        __syncthreads();
    }
    __syncthreads();
    // Write the factored panel back and the dense V (unit diagonal, zeros above).
    for (int e = tid; e < nloc * w; e += kQrThreads) {
        const int r = e / w, j = e - r * w, gr = r0 + r;
        const T v = loc[r * ldl + j];
        A[(int64_t)gr * lda + k + j] = v;
        const int rel = gr - k;
        Vd[(int64_t)rel * kQrW + j] = rel > j ? v : (rel == j ? T(1) : T(0));
    }
    // T of the panel's block reflector, once (CTA 0, warp 0).
    if (cta == 0 && tid < 32) {
        build_t<T>(s_gram, s_tau, w, s_t);
        store_t<T>(s_t, transposed, Tm);
    }
}

// T (or T^T when `transposed`) of a block reflector from the sum of G
// partial Gram matrices (kQrW x kQrW each) and the taus, on one CTA.
template <typename T>
__global__ void larft_kernel(const T *gram_part, int G, const T *tau, int k, int w, T *Tm,
                             int transposed) {
    __shared__ T g[kQrW][kQrW];
    __shared__ T t[kQrW][kQrW];
    __shared__ T taus[kQrW];
    for (int e = threadIdx.x; e < kQrW * kQrW; e += blockDim.x) {
        const int p = e / kQrW, q = e - p * kQrW;
        T s = T(0);
        for (int c = 0; c < G; ++c) s += gram_part[(size_t)c * kQrW * kQrW + p * kQrW + q];
        g[p][q] = s;
    }
    if (threadIdx.x < kQrW) taus[threadIdx.x] = threadIdx.x < w ? tau[k + threadIdx.x] : T(0);
    __syncthreads();
    if (threadIdx.x < 32) {
        build_t<T>(g, taus, w, t);
        store_t<T>(t, transposed, Tm);
    }
}

// ---- the block reflector on a column block C (mk x nc, ldc) ----------------
// C := (I - V T' V^T) C with V (mk x kQrW, ld kQrW) and T' = Tm, in three
// kernels that touch C with VEC-wide accesses (16 bytes) where C allows it:
//   qr_wpart_kernel:  part[g] = V_g^T C_g for row block g (kQrW x nc);
//   qr_wsum_kernel:   W = sum_g part[g], in a fixed order;
//   qr_update_kernel: Y = Tm W in shared memory, then C -= V Y.
// A CTA covers up to kQrUCols columns (blockIdx.y) with kQrUThreads threads.
constexpr int kQrUThreads = 256;
constexpr int kQrUCols = 256;
constexpr int kVtcMaxChunks = 512;  // most row blocks of qr_wpart_kernel
constexpr int kQrRowsInFlight = 8;  // rows of C loaded before any is used

template <typename T, int VEC>
__device__ __forceinline__ void load_vec(const T *p, T (&x)[VEC]) {
    if constexpr (VEC * sizeof(T) == 16) {
        if constexpr (sizeof(T) == 4) {
            const float4 v = *reinterpret_cast<const float4 *>(p);
            x[0] = v.x; x[1] = v.y; x[2] = v.z; x[3] = v.w;
        } else {
            const double2 v = *reinterpret_cast<const double2 *>(p);
            x[0] = v.x; x[1] = v.y;
        }
    } else {
#pragma unroll
        for (int e = 0; e < VEC; ++e) x[e] = p[e];
    }
}

template <typename T, int VEC>
__device__ __forceinline__ void store_vec(T *p, const T (&x)[VEC]) {
    if constexpr (VEC * sizeof(T) == 16) {
        if constexpr (sizeof(T) == 4)
            *reinterpret_cast<float4 *>(p) = make_float4(x[0], x[1], x[2], x[3]);
        else
            *reinterpret_cast<double2 *>(p) = make_double2(x[0], x[1]);
    } else {
#pragma unroll
        for (int e = 0; e < VEC; ++e) p[e] = x[e];
    }
}

// The kQrW entries of V's row r (64- or 128-byte aligned rows).
template <typename T>
__device__ __forceinline__ void load_vrow(const T *V, int64_t r, T (&v)[kQrW]) {
    constexpr int E = 16 / sizeof(T);
    const T *p = V + r * kQrW;
#pragma unroll
    for (int i = 0; i < kQrW; i += E) {
        T x[E];
        load_vec<T, E>(p + i, x);
#pragma unroll
        for (int e = 0; e < E; ++e) v[i + e] = x[e];
    }
}

// Threads split as nq column groups (VEC columns each, nq a power of two
// covering the block's columns, at most kQrUCols / VEC) times ph = 256 / nq
// rows in flight.
// Rows of V staged in shared memory per chunk (double-buffered).
constexpr int kQrVChunk = 128;

// Start copying V rows [cs, min(ce, cs + kQrVChunk)) into vs (16-byte pieces).
template <typename T>
__device__ __forceinline__ void stage_v(const T *V, int cs, int ce, T *vs) {
    const int rows = min(kQrVChunk, ce - cs);
    const int pieces = rows * kQrW * (int)sizeof(T) / 16;
    const unsigned s0 = (unsigned)__cvta_generic_to_shared(vs);
    const char *src = reinterpret_cast<const char *>(V + (int64_t)cs * kQrW);
    for (int i = threadIdx.x; i < pieces; i += kQrUThreads)
        asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s0 + 16u * i),
                     "l"(src + 16 * (int64_t)i)
                     : "memory");
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}

template <typename T>
__device__ __forceinline__ void vrow_smem(const T *vs, int i, T (&v)[kQrW]) {
    constexpr int E = 16 / sizeof(T);
#pragma unroll
    for (int j = 0; j < kQrW; j += E) {
        T x[E];
        load_vec<T, E>(vs + i * kQrW + j, x);
#pragma unroll
        for (int e = 0; e < E; ++e) v[j + e] = x[e];
    }
}

template <typename T, int VEC>
__global__ void __launch_bounds__(kQrUThreads, 2)
    qr_wpart_kernel(const T *V, const T *C, int64_t ldc, int mk, int nc, int rows_per, int nq,
                    T *part) {
    extern __shared__ __align__(16) unsigned char qr_smem[];
    T *red = reinterpret_cast<T *>(qr_smem);  // [ph][kQrW][nq * VEC]
    T *vs = red + kQrW * kQrUThreads * VEC;   // [2][kQrVChunk][kQrW]
    const int ph_n = kQrUThreads / nq, wc = nq * VEC;
    const int q = threadIdx.x % nq, ph = threadIdx.x / nq;
    const int cl = q * VEC, c0 = blockIdx.y * kQrUCols, c = c0 + cl;
    const bool active = c < nc;
    const int r0 = blockIdx.x * rows_per, r1 = min(mk, r0 + rows_per);
    T acc[kQrW][VEC];
#pragma unroll
    for (int j = 0; j < kQrW; ++j)
#pragma unroll
        for (int e = 0; e < VEC; ++e) acc[j][e] = T(0);
    // V in chunks of kQrVChunk rows through shared memory (the next chunk's
    // copy in flight while this one is used); per chunk, kQrRowsInFlight
    // rows' loads of C issued back to back, then used.
    if (r0 < r1) stage_v<T>(V, r0, r1, vs);
    for (int cs = r0, b = 0; cs < r1; cs += kQrVChunk, b ^= 1) {
        const int ce = min(r1, cs + kQrVChunk);
        if (ce < r1) {
            stage_v<T>(V, ce, r1, vs + (b ^ 1) * kQrVChunk * kQrW);
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();
        const T *vb = vs + b * kQrVChunk * kQrW;
        if (active) {
            for (int rb = cs + ph; rb < ce; rb += kQrRowsInFlight * ph_n) {
                T x[kQrRowsInFlight][VEC];
#pragma unroll
                for (int u = 0; u < kQrRowsInFlight; ++u) {
                    const int r = rb + u * ph_n;
                    if (r < ce) {
                        load_vec<T, VEC>(C + (int64_t)r * ldc + c, x[u]);
                    } else {
#pragma unroll
                        for (int e = 0; e < VEC; ++e) x[u][e] = T(0);
                    }
                }
#pragma unroll
                for (int u = 0; u < kQrRowsInFlight; ++u) {
                    const int r = rb + u * ph_n;
                    if (r < ce) {
                        T v[kQrW];
                        vrow_smem<T>(vb, r - cs, v);
#pragma unroll
                        for (int j = 0; j < kQrW; ++j)
#pragma unroll
                            for (int e = 0; e < VEC; ++e) acc[j][e] += v[j] * x[u][e];
                    }
                }
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int j = 0; j < kQrW; ++j)
#pragma unroll
        for (int e = 0; e < VEC; ++e) red[(ph * kQrW + j) * wc + cl + e] = acc[j][e];
    __syncthreads();
    // Sum the row phases in order.
    for (int o = threadIdx.x; o < kQrW * wc; o += kQrUThreads) {
        const int j = o / wc, cc = o - j * wc;
        if (c0 + cc >= nc) continue;
        T t = T(0);
        for (int h = 0; h < ph_n; ++h) t += red[(h * kQrW + j) * wc + cc];
        part[((int64_t)blockIdx.x * kQrW + j) * nc + c0 + cc] = t;
    }
}

// W[j][c] = sum over g of part[g][j][c]: a CTA per (32 columns, j), 8
// lanes over g each summing a fixed residue class, then the lanes in order.
template <typename T>
__global__ void __launch_bounds__(256) qr_wsum_kernel(const T *part, int G, int nc, T *W) {
    __shared__ T s[8][33];
    const int cc = threadIdx.x % 32, lane = threadIdx.x / 32;
    const int c = blockIdx.x * 32 + cc, j = blockIdx.y;
    T t = T(0);
    if (c < nc) {
#pragma unroll 4
        for (int g = lane; g < G; g += 8) t += part[((int64_t)g * kQrW + j) * nc + c];
    }
    s[lane][cc] = t;
    __syncthreads();
    if (lane == 0 && c < nc) {
        T u = T(0);
#pragma unroll
        for (int h = 0; h < 8; ++h) u += s[h][cc];
        W[(int64_t)j * nc + c] = u;
    }
}

template <typename T, int VEC>
__global__ void __launch_bounds__(kQrUThreads, 2)
    qr_update_kernel(const T *V, T *C, int64_t ldc, int mk, int nc, int rows_per, int nq,
                     const T *Tm, const T *W) {
    __shared__ T y[kQrW][kQrUCols];
    __shared__ T tm[kQrW][kQrW];
    const int c0 = blockIdx.y * kQrUCols;
    for (int e = threadIdx.x; e < kQrW * kQrW; e += kQrUThreads) tm[e / kQrW][e % kQrW] = Tm[e];
    __syncthreads();
    // Y = Tm W for this CTA's columns.
    for (int cc = threadIdx.x; cc < kQrUCols; cc += kQrUThreads) {
        T wcol[kQrW];
#pragma unroll
        for (int p = 0; p < kQrW; ++p) wcol[p] = c0 + cc < nc ? W[(int64_t)p * nc + c0 + cc] : T(0);
#pragma unroll
        for (int j = 0; j < kQrW; ++j) {
            T t = T(0);
#pragma unroll
            for (int p = 0; p < kQrW; ++p) t += tm[j][p] * wcol[p];
            y[j][cc] = t;
        }
    }
    __syncthreads();
    extern __shared__ __align__(16) unsigned char qr_smem[];
    T *vs = reinterpret_cast<T *>(qr_smem);  // [2][kQrVChunk][kQrW]
    const int ph_n = kQrUThreads / nq;
    const int q = threadIdx.x % nq, ph = threadIdx.x / nq;
    const int cl = q * VEC, c = c0 + cl;
    const bool active = c < nc;
    T yr[kQrW][VEC];
#pragma unroll
    for (int j = 0; j < kQrW; ++j)
#pragma unroll
        for (int e = 0; e < VEC; ++e) yr[j][e] = active ? y[j][cl + e] : T(0);
    const int r0 = blockIdx.x * rows_per, r1 = min(mk, r0 + rows_per);
    if (r0 < r1) stage_v<T>(V, r0, r1, vs);
    for (int cs = r0, b = 0; cs < r1; cs += kQrVChunk, b ^= 1) {
        const int ce = min(r1, cs + kQrVChunk);
        if (ce < r1) {
            stage_v<T>(V, ce, r1, vs + (b ^ 1) * kQrVChunk * kQrW);
            asm volatile("cp.async.wait_group 1;\n" ::: "memory");
        } else {
            asm volatile("cp.async.wait_group 0;\n" ::: "memory");
        }
        __syncthreads();
        const T *vb = vs + b * kQrVChunk * kQrW;
        if (active) {
            for (int rb = cs + ph; rb < ce; rb += kQrRowsInFlight * ph_n) {
                T x[kQrRowsInFlight][VEC];
#pragma unroll
                for (int u = 0; u < kQrRowsInFlight; ++u) {
                    const int r = rb + u * ph_n;
                    if (r < ce) load_vec<T, VEC>(C + (int64_t)r * ldc + c, x[u]);
                }
#pragma unroll
                for (int u = 0; u < kQrRowsInFlight; ++u) {
                    const int r = rb + u * ph_n;
                    if (r < ce) {
                        T v[kQrW];
                        vrow_smem<T>(vb, r - cs, v);
#pragma unroll
                        for (int j = 0; j < kQrW; ++j)
#pragma unroll
                            for (int e = 0; e < VEC; ++e) x[u][e] -= v[j] * yr[j][e];
                        store_vec<T, VEC>(C + (int64_t)r * ldc + c, x[u]);
                    }
                }
            }
        }
        __syncthreads();
    }
}

// Column groups of a trailing kernel for nc columns at VEC per thread.
static int qr_col_groups(int nc, int vec) {
    const int need = (int)std::min<int64_t>(ceil_div(nc, vec), kQrUCols / vec);
    int nq = 1;
    while (nq < need) nq *= 2;
    return nq;
}

template <typename T>
struct QrRun {
    nmx_ctx ctx;
    cudaStream_t st;
    int m;
    T *Vd, *Tm, *Yk;  // V (m x 16), T (16 x 16), Y (16 x n)
    T *part;          // kVtcMaxChunks x 16 x n partial products
    QrScratch<T> sc;
    size_t panel_smem_max;  // dynamic shared memory the panel kernel may use
};

// Row blocks of the trailing kernels: about `per_sm` CTAs per SM, at least
// 64 rows each.
static int qr_row_blocks(nmx_ctx ctx, int mk, int cb, int per_sm, int *rows_per) {
    int G = (int)std::min<int64_t>({ceil_div(mk, 64), (int64_t)kVtcMaxChunks,
                                    std::max<int64_t>(1, (int64_t)per_sm * ctx->sm_count / cb)});
    G = std::max(G, 1);
    *rows_per = (int)ceil_div(mk, G);
    return (int)ceil_div(mk, *rows_per);
}

// Whether C's rows allow 16-byte accesses at every row start.
template <typename T>
static bool qr_vec_ok(const T *C, int64_t ldc, int nc) {
    constexpr int E = 16 / sizeof(T);
    return (reinterpret_cast<uintptr_t>(C) & 15) == 0 && ldc % E == 0 && nc % E == 0;
}

// W = V^T C (kQrW x nc, into Wout) for the mk x nc block C.
template <typename T>
static int vtc(QrRun<T> &R, int mk, const T *C, int64_t ldc, int nc, T *Wout) {
    constexpr int E = 16 / sizeof(T);
    const int cb = (int)ceil_div(nc, kQrUCols);
    int rows_per = 0;
    const int G = qr_row_blocks(R.ctx, mk, cb, 2, &rows_per);
    // Shared memory of the phase sums: ph x kQrW x (nq VEC) = kQrW x 256 VEC values.
    if (qr_vec_ok(C, ldc, nc)) {
        const int nq = qr_col_groups(nc, E);
        const size_t smem = sizeof(T) * ((size_t)kQrW * kQrUThreads * E + 2 * kQrVChunk * kQrW);
        qr_wpart_kernel<T, E><<<dim3(G, cb), kQrUThreads, smem, R.st>>>(R.Vd, C, ldc, mk, nc,
                                                                          rows_per, nq, R.part);
    } else {
        const int nq = qr_col_groups(nc, 1);
        const size_t smem = sizeof(T) * ((size_t)kQrW * kQrUThreads + 2 * kQrVChunk * kQrW);
        qr_wpart_kernel<T, 1><<<dim3(G, cb), kQrUThreads, smem, R.st>>>(R.Vd, C, ldc, mk, nc,
                                                                          rows_per, nq, R.part);
    }
    qr_wsum_kernel<T><<<dim3((unsigned)ceil_div(nc, 32), kQrW), 256, 0, R.st>>>(R.part, G, nc, Wout);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

// Factor the panel at column k (width w) and record V and T' for it.
template <typename T>
static int qr_panel(QrRun<T> &R, T *A, int64_t lda, T *tau, int k, int w, int transposed) {
    const int mk = R.m - k;
    int G = (int)std::min<int64_t>(std::min(R.ctx->sm_count, kQrMaxG), ceil_div(mk, 64));
    G = std::max(G, 1);
    int rpc = (int)ceil_div(mk, G);
    G = (int)ceil_div(mk, rpc);
    const size_t smem = sizeof(T) * (size_t)rpc * (kQrW + 1);
    if (smem > R.panel_smem_max) {
        set_error("QR panel of %d rows does not fit the cooperative grid", mk);
        return NMX_ERR_UNSUPPORTED;
    }
    NMX_CUDA_TRY(cudaMemsetAsync(R.sc.bar, 0, sizeof(unsigned), R.st));
    NMX_CUDA_TRY(cudaMemsetAsync(R.Vd, 0, sizeof(T) * (size_t)mk * kQrW, R.st));
    void *args[] = {&A, &lda, &R.m, &k, &w, &rpc, &tau, &R.Vd, &R.Tm, &transposed, &R.sc};
    NMX_CUDA_TRY(cudaLaunchCooperativeKernel((void *)geqr2_coop_kernel<T>, dim3(G), dim3(kQrThreads),
                                             args, smem, R.st));
    return 0;
}

// C := (I - V T' V^T) C for C = rows [k, m) x cols [c0, c1) of Cm.
template <typename T>
static int apply_reflector(QrRun<T> &R, int k, T *Cm, int64_t ldc, int c0, int c1) {
    constexpr int E = 16 / sizeof(T);
    const int nc = c1 - c0, mk = R.m - k;
    if (nc <= 0) return 0;
    T *C = Cm + (int64_t)k * ldc + c0;
    // W = V^T C, then Y = T' W and C -= V Y.
    NMX_TRY(vtc<T>(R, mk, C, ldc, nc, R.Yk));
    const int cb = (int)ceil_div(nc, kQrUCols);
    int rows_per = 0;
    const int G = qr_row_blocks(R.ctx, mk, cb, 4, &rows_per);
    const size_t vsm = sizeof(T) * 2 * kQrVChunk * kQrW;
    if (qr_vec_ok(C, ldc, nc))
        qr_update_kernel<T, E><<<dim3(G, cb), kQrUThreads, vsm, R.st>>>(
            R.Vd, C, ldc, mk, nc, rows_per, qr_col_groups(nc, E), R.Tm, R.Yk);
    else
        qr_update_kernel<T, 1><<<dim3(G, cb), kQrUThreads, vsm, R.st>>>(
            R.Vd, C, ldc, mk, nc, rows_per, qr_col_groups(nc, 1), R.Tm, R.Yk);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

template <typename T>
static int qr_setup(nmx_ctx ctx, cudaStream_t st, int64_t m, int64_t n, QrRun<T> &R) {
    const int G = ctx->sm_count;
    const size_t nn = (size_t)std::max<int64_t>(n, kQrW);
    size_t elems = (size_t)m * kQrW + kQrW * kQrW + (size_t)kQrW * nn +
                   (size_t)kVtcMaxChunks * kQrW * nn + 2 * (size_t)kQrVec * kQrPart +
                   (size_t)kQrW * kQrW + 64;
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
    R.sc.gram_part = R.sc.part + 2 * (size_t)kQrVec * kQrPart;
    R.sc.bar = reinterpret_cast<unsigned *>(R.sc.gram_part + (size_t)kQrW * kQrW);
    R.sc.err = reinterpret_cast<int *>(R.sc.bar + 1);
    NMX_CUDA_TRY(cudaMemsetAsync(R.sc.err, 0, sizeof(int), st));
    cudaFuncAttributes fa;
    NMX_CUDA_TRY(cudaFuncGetAttributes(&fa, geqr2_coop_kernel<T>));
    R.panel_smem_max = ctx->smem_optin - fa.sharedSizeBytes;
    NMX_CUDA_TRY(cudaFuncSetAttribute(geqr2_coop_kernel<T>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)R.panel_smem_max));
    constexpr int E = 16 / sizeof(T);
    NMX_CUDA_TRY(cudaFuncSetAttribute(
        qr_wpart_kernel<T, E>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)(sizeof(T) * ((size_t)kQrW * kQrUThreads * E + 2 * kQrVChunk * kQrW))));
    NMX_CUDA_TRY(cudaFuncSetAttribute(
        qr_wpart_kernel<T, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize,
        (int)(sizeof(T) * ((size_t)kQrW * kQrUThreads + 2 * kQrVChunk * kQrW))));
    NMX_CUDA_TRY(cudaFuncSetAttribute(qr_update_kernel<T, E>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(sizeof(T) * 2 * kQrVChunk * kQrW)));
    NMX_CUDA_TRY(cudaFuncSetAttribute(qr_update_kernel<T, 1>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(sizeof(T) * 2 * kQrVChunk * kQrW)));
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
        NMX_TRY(vtc<T>(R, (int)mk, R.Vd, kQrW, kQrW, R.sc.gram_part));
        larft_kernel<T><<<1, 256, 0, st>>>(R.sc.gram_part, 1, tau, k, w, R.Tm, 0);
        NMX_CUDA_TRY(cudaGetLastError());
        rc = apply_reflector<T>(R, k, Q, ldq, k, (int)n);
        if (rc) return rc;
    }
    return 0;
}

// B := Q B for the m x ncols block B (ldb), Q = H_0 ... H_{k-1} from
// reflectors stored as geqrf leaves them in F (m x k, ldf): orgqr's replay,
// last panel first, on B instead of the identity.  The symmetric
// eigensolver forms its eigenvectors Q Z with it.
int qr_apply_q_f64(nmx_ctx ctx, cudaStream_t st, int64_t m, int64_t k, const double *F,
                   int64_t ldf, const double *tau, double *B, int64_t ldb, int64_t ncols) {
    if (k <= 0 || ncols <= 0) return 0;
    QrRun<double> R;
    NMX_TRY(qr_setup<double>(ctx, st, m, std::max<int64_t>(k, ncols), R));
    const int steps = (int)ceil_div(k, kQrW);
    for (int s = 0; s < steps; ++s) {
        const int kk = (steps - 1 - s) * kQrW;
        const int w = (int)std::min<int64_t>(kQrW, k - kk);
        const int64_t mk = m - kk;
        pack_v_kernel<double><<<(unsigned)ceil_div(mk * kQrW, 256), 256, 0, st>>>(
            F, ldf, (int)m, kk, w, R.Vd, nullptr);
        NMX_CUDA_TRY(cudaGetLastError());
        NMX_TRY(vtc<double>(R, (int)mk, R.Vd, kQrW, kQrW, R.sc.gram_part));
        larft_kernel<double><<<1, 256, 0, st>>>(R.sc.gram_part, 1, tau, kk, w, R.Tm, 0);
        NMX_CUDA_TRY(cudaGetLastError());
        NMX_TRY(apply_reflector<double>(R, kk, B, ldb, 0, (int)ncols));
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
        NMX_TRY(vtc<T>(R, (int)mk, R.Vd, kQrW, kQrW, R.sc.gram_part));
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
