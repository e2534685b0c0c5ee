// Symmetric eigendecomposition of one n x n matrix on the device (sm_100a):
// numax's Tensor-tier eigh / eigvalsh (numax/linalg/eigen.mojo:1268-1341,
// 1449+): eigenvalues ascending, orthonormal eigenvectors as columns, only
// the lower triangle read.
//
// numax reduces A to tridiagonal form (sytrd), runs implicit QL on the host
// with its rotations batched into device GEMMs, sorts on the host and forms
// Q Z with one more GEMM.  Here every step is on the device:
//   1. sym_lower_kernel: the lower triangle mirrored into a full FP64 work
//      copy (tiled transpose), and max |a_ij| for a power-of-two scaling.
//   2. latrd_kernel: Householder tridiagonalization by 32-column panels,
//      each panel ONE cooperative launch with two grid rounds per column
//      (the column's norm; then W^T v, V^T v and y . v in one vector), the
//      trailing matrix read once per column for y = A22 v (v staged in
//      shared memory by chunks) and updated once per panel,
//      A -= V W^T + W V^T, on the library's FP64 GEMM.  Reflectors stay
//      below the subdiagonal in LAPACK's lower layout, numax's beta/tau
//      convention.
//   3. eigenvalues only: Sturm-count bisection, one thread per eigenvalue.
//      Eigenvectors: divide and conquer on the tridiagonal (tridiag_dc.cuh):
//      level by level, every merge of a level at once -- deflation, secular
//      roots, Loewner z-hat, the eigenvector matrix, Q_new = Q_sel U on the
//      library's FP64 GEMM, the merged order by ranks.
//   4. Q Z by the QR module's block reflectors (16-column panels), last
//      panel first, on Z's rows 1..n-1.
// numax's QL and this divide and conquer give the same eigenvalues to
// rounding and the same eigenvectors up to sign (and up to a basis of each
// multiple eigenvalue's space).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

#include "dense_common.cuh"
#include "tridiag_dc.cuh"

namespace nmx {

// B := Q B (QR-style reflectors in F, m x k): dense_qr.cu.
int qr_apply_q_f64(nmx_ctx ctx, cudaStream_t st, int64_t m, int64_t k, const double *F,
                   int64_t ldf, const double *tau, double *B, int64_t ldb, int64_t ncols);

namespace {

constexpr int kTrdThreads = 512;
constexpr int kTrdWarps = kTrdThreads / 32;
constexpr int kTrdRows = 8;      // rows a warp owns at most: n - 1 <= 8 x warps in the grid
constexpr int kTrdChunk = 4096;  // columns of v staged in shared memory at once

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// ---- 1. symmetric work copy --------------------------------------------------

// W (ld ldw) = the symmetric matrix whose lower triangle is A's; *maxabs
// receives max |a_ij| over the lower triangle as the bits of a non-negative
// double (+infinity when the triangle holds a NaN or an infinity).
template <typename T>
__global__ void sym_lower_kernel(const T *A, int64_t lda, int n, double *W, int64_t ldw,
                                 unsigned long long *maxabs) {
    __shared__ double tile[32][33];
    const int tx = blockIdx.x, ty = blockIdx.y;
    if (tx > ty) return;
    const int lx = threadIdx.x & 31, ly = threadIdx.x >> 5;  // 32 x 8 threads
    double m = 0.0;
    bool bad = false;
    for (int i = ly; i < 32; i += 8) {
        const int r = ty * 32 + i, c = tx * 32 + lx;
        double v = 0.0;
        if (r < n && c < n && c <= r) {
            v = (double)A[(int64_t)r * lda + c];
            m = fmax(m, fabs(v));
            bad |= !(fabs(v) <= 1.7976931348623157e308);
        }
        tile[i][lx] = v;
    }
    if (bad) m = __longlong_as_double(0x7ff0000000000000ll);  // +inf marks a NaN or an infinity
    __syncthreads();
    for (int i = ly; i < 32; i += 8) {
        const int r = ty * 32 + i, c = tx * 32 + lx;
        if (r < n && c < n) {
            // Below the diagonal (or on it) as read; above it (diagonal tile
            // only), the mirror from the same tile.
            W[(int64_t)r * ldw + c] = (c <= r) ? tile[i][lx] : tile[lx][i];
        }
        const int rt = tx * 32 + i, ct = ty * 32 + lx;  // the transposed tile
        if (tx != ty && rt < n && ct < n) W[(int64_t)rt * ldw + ct] = tile[lx][i];
    }
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 16));
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 8));
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 4));
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 2));
    m = fmax(m, __shfl_xor_sync(0xffffffffu, m, 1));
    if (lx == 0 && m != 0.0) atomicMax(maxabs, (unsigned long long)__double_as_longlong(m));
}

// ---- 2. tridiagonalization ---------------------------------------------------

constexpr int kLrdNb = 32;              // panel width (columns per launch)
constexpr int kLrdVec = 2 * kLrdNb + 1;  // W^T v, V^T v and y . v: one round's sums
constexpr int kLrdSub = 7;              // threads per value in the cross-CTA sum (65 x 7 <= 512)

struct LrdArgs {
    double *A;  // the symmetric work matrix (full storage), scaled
    int64_t lda;
    int n;
    int p, jb;            // the panel: columns [p, p + jb)
    double *d, *e, *tau;  // diagonal, subdiagonal, reflector scales
    double *Vp, *Wp;      // [n][kLrdNb] the panel's v and w, row-major
    double *xbuf;         // [n] the current column, brought up to date
    double *ybuf;         // [n] A22 v of the current column
    double *part;         // [2][kLrdVec][G] per-CTA partial sums (double-buffered)
    unsigned *bar;
    int *err;
};

// One grid round over a vector of `nv` sums: the CTA's threads have added
// their values into red[warp][v]; every CTA publishes its totals, and after
// the barrier sums all CTAs' in the same fixed order into out[0 .. nv).
// Returns false if the barrier gave up.
__device__ bool lrd_round(const LrdArgs &a, unsigned &gen, int nv, double (*red)[kLrdVec],
                          double *sub, double *out, int *s_flag) {
    const int G = gridDim.x;
    __syncthreads();
    double *slot = a.part + (size_t)(gen & 1) * kLrdVec * G;
    if (threadIdx.x < nv) {
        double t = 0.0;
        for (int w = 0; w < kTrdWarps; ++w) t += red[w][threadIdx.x];
        slot[(size_t)threadIdx.x * G + blockIdx.x] = t;
    }
    if (!grid_barrier(a.bar, gen++, (unsigned)G, a.err, s_flag)) return false;
    if (threadIdx.x < nv * kLrdSub) {
        const int v = threadIdx.x / kLrdSub, s = threadIdx.x - v * kLrdSub;
        const double *src = slot + (size_t)v * G;
        double t = 0.0;
        for (int g = s; g < G; g += kLrdSub) t += __ldcg(src + g);
        sub[threadIdx.x] = t;
    }
    __syncthreads();
    if (threadIdx.x < nv) {
        double t = 0.0;
        for (int s = 0; s < kLrdSub; ++s) t += sub[threadIdx.x * kLrdSub + s];
        out[threadIdx.x] = t;
    }
    __syncthreads();
    return true;
}

// One panel of the Householder reduction to tridiagonal form (LAPACK's
// latrd, lower), in one cooperative launch: the trailing matrix stays as it
// was at the panel's start and each column is brought up to date with the
// panel's earlier reflectors through V and W,
//   a = A[:, j] - V W[j, :]^T - W V[j, :]^T                   (round 1: |x|)
//   beta = -sign(alpha) |x| (alpha <= 0 gives +|x|), tau = (beta - alpha)/beta,
//   v = (1, x[1:] / (alpha - beta))
//   y = A22 v; sums W^T v, V^T v, y . v                       (round 2)
//   w = tau (y - V (W^T v) - W (V^T v)) - (tau/2)(w . v) v,
// with w . v = tau (y . v - 2 (W^T v) . (V^T v)).  The caller then updates
// the trailing matrix with A -= V W^T + W V^T on the GEMM.  Row r belongs to
// warp r mod (warps in the grid); the reflector goes below the subdiagonal
// of column j, beta to the subdiagonal.
__global__ void __launch_bounds__(kTrdThreads, 1) latrd_kernel(LrdArgs a) {
    __shared__ double sv[kTrdChunk];
    __shared__ double red[kTrdWarps][kLrdVec];
    __shared__ double sub[kLrdVec * kLrdSub];
    __shared__ double tot[kLrdVec];
    __shared__ double s_vj[kLrdNb], s_wj[kLrdNb];  // row j of V and W
    __shared__ double s_t1[kLrdNb], s_t2[kLrdNb];  // the previous column's W^T v, V^T v
    __shared__ int s_flag;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int NW = gridDim.x * kTrdWarps, gw = blockIdx.x * kTrdWarps + warp;
    const int n = a.n, p = a.p;
    const int64_t lda = a.lda;
    const double *A = a.A;
    unsigned gen = 0;
    double tau_prev = 0.0, aw_prev = 0.0;

    for (int i = 0; i < a.jb; ++i) {
        const int j = p + i;
        // Row j of the panel's V and W: earlier columns from memory; the
        // previous column's w_j computed here (its owner wrote it after the
        // last barrier).
        if (threadIdx.x < 32) {
            const int t = lane;
            double vj = 0.0, wj = 0.0;
            if (t < i) vj = __ldcg(a.Vp + (size_t)j * kLrdNb + t);
            if (t + 1 < i) wj = __ldcg(a.Wp + (size_t)j * kLrdNb + t);
            double corr = 0.0;
            if (t + 1 < i) corr = vj * s_t1[t] + wj * s_t2[t];
            corr = warp_sum(corr);
            if (i > 0 && t == i - 1)
                wj = tau_prev * (__ldcg(a.ybuf + j) - corr) + aw_prev * vj;
            s_vj[t] = vj;
            s_wj[t] = wj;
        }
        __syncthreads();

        // The column brought up to date on the owned rows r >= j.
        double pn = 0.0;
        int r0 = gw;
        if (r0 < j) r0 += ((j - r0 + NW - 1) / NW) * NW;
        for (int r = r0; r < n; r += NW) {
            double c = 0.0;
            if (lane < i)
                c = a.Vp[(size_t)r * kLrdNb + lane] * s_wj[lane] +
                    a.Wp[(size_t)r * kLrdNb + lane] * s_vj[lane];
            c = warp_sum(c);
            const double x = A[(int64_t)r * lda + j] - c;
            if (lane == 0) {
                if (r == j) a.d[j] = x;
                if (r >= j + 1) a.xbuf[r] = x;
                if (r >= j + 2) pn += x * x;
            }
        }
        if (lane == 0) red[warp][0] = pn;  // lane 0 holds the warp's rows
        if (!lrd_round(a, gen, 1, red, sub, tot, &s_flag)) return;
        const double xn2 = tot[0];

        const double alpha = __ldcg(a.xbuf + j + 1);
        double beta, tau, scale;
        if (xn2 == 0.0) {
            beta = alpha;
            tau = 0.0;
            scale = 0.0;
        } else {
            const double nrm = sqrt(alpha * alpha + xn2);
            beta = alpha <= 0.0 ? nrm : -nrm;
            tau = (beta - alpha) / beta;
            scale = 1.0 / (alpha - beta);
        }
        if (blockIdx.x == 0 && threadIdx.x == 0) {
            a.e[j] = beta;
            a.tau[j] = tau;
        }

        // y = A22 v on the owned rows (v staged by chunks), with the sums.
        r0 = gw;
        if (r0 < j + 1) r0 += ((j + 1 - r0 + NW - 1) / NW) * NW;
        double acc[kTrdRows];
#pragma unroll
        for (int t = 0; t < kTrdRows; ++t) acc[t] = 0.0;
        for (int c0 = j + 1; c0 < n; c0 += kTrdChunk) {
            const int cn = min(kTrdChunk, n - c0);
            __syncthreads();
            for (int c = threadIdx.x; c < cn; c += kTrdThreads) {
                const int cc = c0 + c;
                sv[c] = cc == j + 1 ? 1.0 : __ldcg(a.xbuf + cc) * scale;
            }
            __syncthreads();
#pragma unroll
            for (int t = 0; t < kTrdRows; ++t) {
                const int r = r0 + t * NW;
                if (r >= n) break;
                const double *row = A + (int64_t)r * lda + c0;
                // Eight loads in flight per lane before any is used.
                double s[8] = {0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
                int c = lane;
                for (; c + 224 < cn; c += 256) {
                    double x[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) x[u] = row[c + 32 * u];
#pragma unroll
                    for (int u = 0; u < 8; ++u) s[u] = fma(x[u], sv[c + 32 * u], s[u]);
                }
                for (; c < cn; c += 32) s[0] = fma(row[c], sv[c], s[0]);
                acc[t] += ((s[0] + s[1]) + (s[2] + s[3])) + ((s[4] + s[5]) + (s[6] + s[7]));
            }
        }
        double t1 = 0.0, t2 = 0.0, yv = 0.0;  // lane t: W[:, t]^T v, V[:, t]^T v
        double yr[kTrdRows], vr[kTrdRows];
#pragma unroll
        for (int t = 0; t < kTrdRows; ++t) {
            const int r = r0 + t * NW;
            yr[t] = vr[t] = 0.0;
            if (r >= n) break;
            const double y = warp_sum(acc[t]);
            const double v = r == j + 1 ? 1.0 : __ldcg(a.xbuf + r) * scale;
            yr[t] = y;
            vr[t] = v;
            yv += y * v;
            if (lane < i) {
                t1 += a.Wp[(size_t)r * kLrdNb + lane] * v;
                t2 += a.Vp[(size_t)r * kLrdNb + lane] * v;
            }
            if (lane == 0) {
                a.ybuf[r] = y;
                a.Vp[(size_t)r * kLrdNb + i] = v;
                a.A[(int64_t)r * lda + j] = r == j + 1 ? beta : v;  // the reflector's storage
            }
        }
        // The round's vector holds only what is nonzero: W^T v (i values),
        // V^T v (i values), y . v.
        if (lane < i) {
            red[warp][lane] = t1;
            red[warp][i + lane] = t2;
        }
        if (lane == 0) red[warp][2 * i] = yv;
        if (!lrd_round(a, gen, 2 * i + 1, red, sub, tot, &s_flag)) return;
        if (threadIdx.x < kLrdNb) {
            const double u1 = threadIdx.x < i ? tot[threadIdx.x] : 0.0;
            const double u2 = threadIdx.x < i ? tot[i + threadIdx.x] : 0.0;
            const double yvt = tot[2 * i];
            __syncwarp();
            tot[threadIdx.x] = u1;
            tot[kLrdNb + threadIdx.x] = u2;
            if (threadIdx.x == 0) tot[2 * kLrdNb] = yvt;
        }
        __syncthreads();

        // w on the owned rows.
        double t12 = 0.0;
        for (int t = 0; t < i; ++t) t12 += tot[t] * tot[kLrdNb + t];
        const double aw = -0.5 * tau * tau * (tot[2 * kLrdNb] - 2.0 * t12);
#pragma unroll
        for (int t = 0; t < kTrdRows; ++t) {
            const int r = r0 + t * NW;
            if (r >= n) break;
            double c = 0.0;
            if (lane < i)
                c = a.Vp[(size_t)r * kLrdNb + lane] * tot[lane] +
                    a.Wp[(size_t)r * kLrdNb + lane] * tot[kLrdNb + lane];
            c = warp_sum(c);
            if (lane == 0) a.Wp[(size_t)r * kLrdNb + i] = tau * (yr[t] - c) + aw * vr[t];
        }
        if (threadIdx.x < kLrdNb) {
            s_t1[threadIdx.x] = tot[threadIdx.x];
            s_t2[threadIdx.x] = tot[kLrdNb + threadIdx.x];
        }
        tau_prev = tau;
        aw_prev = aw;
        __syncthreads();
    }
}

// The trailing 2 x 2 (or 1 x 1) once every panel's update is in.
__global__ void trd_tail_kernel(const double *A, int64_t lda, int n, double *d, double *e,
                                double *tau) {
    if (threadIdx.x != 0) return;
    if (n == 1) {
        d[0] = A[0];
        return;
    }
    d[n - 2] = A[(int64_t)(n - 2) * lda + n - 2];
    d[n - 1] = A[(int64_t)(n - 1) * lda + n - 1];
    e[n - 2] = A[(int64_t)(n - 1) * lda + n - 2];
    tau[n - 2] = 0.0;
}

// A *= 2^-ex (exact), ex from max |a_ij|, so the sums of squares stay in range.
__global__ void scale_kernel(double *A, int64_t n2, int ex) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n2) A[e] = ldexp(A[e], -ex);
}

// ---- 3a. eigenvalues by bisection --------------------------------------------

// Eigenvalue k (ascending) of the tridiagonal (d, e): dc::sturm_kth's
// multisection on the Sturm count inside the Gershgorin interval (widened
// by the rounding of the counts), scaled back by 2^scale_exp.
template <typename T>
__global__ void bisect_kernel(int n, const double *d, const double *e, const int *scale_exp,
                              T *W) {
    const int k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n) return;
    double lo = d[0], hi = d[0], emax2 = 0.0;
    for (int i = 0; i < n; ++i) {
        const double r = (i > 0 ? fabs(e[i - 1]) : 0.0) + (i + 1 < n ? fabs(e[i]) : 0.0);
        lo = fmin(lo, d[i] - r);
        hi = fmax(hi, d[i] + r);
        if (i + 1 < n) emax2 = fmax(emax2, e[i] * e[i]);
    }
    const double pivmin = 2.2250738585072014e-308 * fmax(1.0, emax2);
    const double tnorm = fmax(fabs(lo), fabs(hi));
    lo -= 2.0 * dc::kEps * tnorm * n + pivmin;
    hi += 2.0 * dc::kEps * tnorm * n + pivmin;
    W[k] = (T)ldexp(dc::sturm_kth(n, d, e, k, lo, hi, pivmin), *scale_exp);
}

// ---- 3b. divide and conquer --------------------------------------------------

struct DcBuf {
    double *D;                  // [n] eigenvalues of the current blocks
    double *e;                  // [n] the (normalized) off-diagonal: the tear couplings
    double *rho;                // [merges] 2 |beta|
    int *kc;                    // [merges][3] k, ndef, nrot
    double *zvec, *ds, *zs, *dl, *zl, *ddef, *rc, *rs, *tau, *zhat;  // [n] each
    int *perm, *cnd, *cdef, *ra, *rb, *org, *slot;                    // [n] each
    double *Qa;                 // [n x n] eigenvectors of the blocks, merged in place
    double *Qsel, *Ut, *Qout;   // [n x mmax] per-level products
    double *norm;               // [1] the tridiagonal's scale
    int4 *merges;               // (lo, mid, hi, -) of every merge, level by level
};

// max(|d_i|, |e_i|) of the tridiagonal into *norm (one CTA).
__global__ void dc_norm_kernel(int n, const double *d, const double *e, double *norm) {
    __shared__ double red[32];
    double m = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        m = fmax(m, fabs(d[i]));
        if (i + 1 < n) m = fmax(m, fabs(e[i]));
    }
    for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t = fmax(t, red[w]);
        *norm = t > 0.0 ? t : 1.0;
    }
}

// D = d / norm less the tears' |beta| on the two entries each couples;
// e = e / norm; Qa = I.
__global__ void dc_init_kernel(int n, const double *d, const double *e, const unsigned char *split,
                               const double *norm, double *D, double *en, double *Qa) {
    const int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (idx < (int64_t)n * n) {
        const int r = (int)(idx / n), c = (int)(idx - (int64_t)r * n);
        Qa[idx] = r == c ? 1.0 : 0.0;
    }
    if (idx < n) {
        const int i = (int)idx;
        const double s = 1.0 / *norm;
        double v = d[i] * s;
        if (i > 0 && split[i]) v -= fabs(e[i - 1] * s);
        if (i + 1 < n && split[i + 1]) v -= fabs(e[i] * s);
        D[i] = v;
        en[i] = i + 1 < n ? e[i] * s : 0.0;
    }
}

// Per merge: z from the halves' boundary rows of Qa, then the deflation pass
// (one thread: it is sequential).
__global__ void dc_deflate_kernel(const int4 *merges, int n, DcBuf b) {
    const int4 mg = merges[blockIdx.x];
    const int lo = mg.x, mid = mg.y, hi = mg.z, m = hi - lo, m1 = mid - lo;
    const double beta = b.e[mid - 1];
    const double sg = beta < 0.0 ? -1.0 : 1.0;
    const double inv_sqrt2 = 0.70710678118654752440;
    for (int i = threadIdx.x; i < m; i += blockDim.x)
        b.zvec[lo + i] = i < m1 ? b.Qa[(int64_t)(mid - 1) * n + lo + i] * inv_sqrt2
                                : sg * b.Qa[(int64_t)mid * n + lo + i] * inv_sqrt2;
    __syncthreads();
    if (threadIdx.x != 0) return;
    const double rho = 2.0 * fabs(beta);
    const dc::Deflation r =
        dc::deflate(m, m1, b.D + lo, b.zvec + lo, rho, b.perm + lo, b.ds + lo, b.zs + lo, b.dl + lo,
                    b.zl + lo, b.cnd + lo, b.ddef + lo, b.cdef + lo, b.ra + lo, b.rb + lo,
                    b.rc + lo, b.rs + lo);
    b.rho[blockIdx.x] = rho;
    b.kc[3 * blockIdx.x] = r.k;
    b.kc[3 * blockIdx.x + 1] = r.ndef;
    b.kc[3 * blockIdx.x + 2] = r.nrot;
}

// Zero the off-halves blocks of each merge's Q block (warp per row), then
// apply the merge's rotations to the row (lane 0; they are sequential).
__global__ void dc_rotate_kernel(const int4 *merges, int n, DcBuf b) {
    const int4 mg = merges[blockIdx.y];
    const int lo = mg.x, mid = mg.y, hi = mg.z;
    const int i = lo + blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (i >= hi) return;
    double *row = b.Qa + (int64_t)i * n;
    const int z0 = i < mid ? mid : lo, z1 = i < mid ? hi : mid;
    for (int c = z0 + lane; c < z1; c += 32) row[c] = 0.0;
    __syncwarp();
    if (lane != 0) return;
    const int nrot = b.kc[3 * blockIdx.y + 2];
    for (int t = 0; t < nrot; ++t) {
        double &x = row[lo + b.ra[lo + t]];
        double &y = row[lo + b.rb[lo + t]];
        const double c = b.rc[lo + t], s = b.rs[lo + t];
        const double xn = c * x + s * y, yn = c * y - s * x;
        x = xn;
        y = yn;
    }
}

__global__ void dc_secular_kernel(const int4 *merges, DcBuf b) {
    const int lo = merges[blockIdx.y].x;
    const int k = b.kc[3 * blockIdx.y];
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= k) return;
    int o;
    double t;
    dc::secular_root(k, b.dl + lo, b.zl + lo, b.rho[blockIdx.y], j, &o, &t);
    b.org[lo + j] = o;
    b.tau[lo + j] = t;
}

__global__ void dc_zhat_kernel(const int4 *merges, DcBuf b) {
    const int lo = merges[blockIdx.y].x;
    const int k = b.kc[3 * blockIdx.y];
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= k) return;
    b.zhat[lo + i] =
        dc::lowner_z(k, b.dl + lo, b.zl + lo, b.rho[blockIdx.y], b.org + lo, b.tau + lo, i);
}

// Ut row j (eigenvector j of D + rho z z^T): z-hat_i / (d_i - lambda_j),
// normalized.  One CTA per j.
__global__ void dc_vec_kernel(const int4 *merges, int mmax, DcBuf b) {
    __shared__ double red[32];
    const int lo = merges[blockIdx.y].x;
    const int k = b.kc[3 * blockIdx.y];
    const int j = blockIdx.x;
    if (j >= k) return;
    const double *dl = b.dl + lo;
    const int o = b.org[lo + j];
    const double t = b.tau[lo + j];
    double *u = b.Ut + (int64_t)lo * mmax + (int64_t)j * k;
    double s = 0.0;
    for (int i = threadIdx.x; i < k; i += blockDim.x) {
        const double v = b.zhat[lo + i] / dc::delta_ij(dl, i, o, t);
        u[i] = v;
        s += v * v;
    }
    s = warp_sum(s);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        double v = threadIdx.x < (blockDim.x >> 5) ? red[threadIdx.x] : 0.0;
        v = warp_sum(v);
        if (threadIdx.x == 0) red[0] = 1.0 / sqrt(v);
    }
    __syncthreads();
    const double inv = red[0];
    for (int i = threadIdx.x; i < k; i += blockDim.x) u[i] *= inv;
}

// Qsel (m x m) = the merge's Q block with its columns reordered: the k
// surviving ones first, then the deflated ones.
__global__ void dc_gather_kernel(const int4 *merges, int n, int mmax, DcBuf b) {
    const int4 mg = merges[blockIdx.y];
    const int lo = mg.x, m = mg.z - mg.x;
    const int k = b.kc[3 * blockIdx.y];
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)m * m) return;
    const int i = (int)(e / m), t = (int)(e - (int64_t)i * m);
    const int col = t < k ? b.cnd[lo + t] : b.cdef[lo + t - k];
    b.Qsel[(int64_t)lo * mmax + e] = b.Qa[(int64_t)(lo + i) * n + lo + col];
}

// Qout (m x k) = Qsel[:, :k] Ut^T for merges too small for the GEMM (one
// CTA each).
__global__ void dc_small_gemm_kernel(const int4 *merges, int mmax, DcBuf b) {
    const int4 mg = merges[blockIdx.x];
    const int lo = mg.x, m = mg.z - mg.x;
    const int k = b.kc[3 * blockIdx.x];
    const double *Qs = b.Qsel + (int64_t)lo * mmax;
    const double *U = b.Ut + (int64_t)lo * mmax;
    double *Qo = b.Qout + (int64_t)lo * mmax;
    for (int e = threadIdx.x; e < m * k; e += blockDim.x) {
        const int i = e / k, j = e - i * k;
        double s = 0.0;
        for (int t = 0; t < k; ++t) s = fma(Qs[i * m + t], U[j * k + t], s);
        Qo[e] = s;
    }
}

// The merged eigenvalues in ascending order: slot[lo + rank] = candidate.
__global__ void dc_rank_kernel(const int4 *merges, DcBuf b) {
    const int4 mg = merges[blockIdx.y];
    const int lo = mg.x, m = mg.z - mg.x;
    const int k = b.kc[3 * blockIdx.y], ndef = b.kc[3 * blockIdx.y + 1];
    const int c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= m) return;
    const int r =
        dc::merged_rank(k, ndef, b.dl + lo, b.org + lo, b.tau + lo, b.ddef + lo, c);
    b.slot[lo + r] = c;
    b.D[lo + r] = c < k ? b.dl[lo + b.org[lo + c]] + b.tau[lo + c] : b.ddef[lo + c - k];
}

// The merged block of Qa in the ascending order (warp per row): a root's
// column from Qout, a deflated one from Qsel.
__global__ void dc_write_kernel(const int4 *merges, int n, int mmax, DcBuf b) {
    const int4 mg = merges[blockIdx.y];
    const int lo = mg.x, m = mg.z - mg.x;
    const int k = b.kc[3 * blockIdx.y];
    const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (i >= m) return;
    const double *qo = b.Qout + (int64_t)lo * mmax + (int64_t)i * k;
    const double *qs = b.Qsel + (int64_t)lo * mmax + (int64_t)i * m;
    double *qa = b.Qa + (int64_t)(lo + i) * n + lo;
    for (int q = threadIdx.x & 31; q < m; q += 32) {
        int s = b.slot[lo + q];
        s = (s >= 0 && s < m) ? s : 0;  // ranks are a permutation of 0..m-1
        qa[q] = s < k ? qo[s] : qs[s];
    }
}

template <typename T>
__global__ void dc_finish_kernel(int n, const double *D, const double *norm, const int *scale_exp,
                                 T *W) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) W[i] = (T)ldexp(D[i] * *norm, *scale_exp);
}

template <typename T>
__global__ void copy_out_kernel(const double *Z, int n, T *V, int64_t ldv) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)n * n) return;
    const int r = (int)(e / n), c = (int)(e - (int64_t)r * n);
    V[(int64_t)r * ldv + c] = (T)Z[e];
}

// A matrix holding a NaN or an infinity: info = 1 and NaN outputs.
template <typename T>
__global__ void nonfinite_kernel(int n, T *W, T *V, int64_t ldv, int32_t *info) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    const T nan = (T)__longlong_as_double(0x7ff8000000000000ll);
    if (e == 0) *info = 1;
    if (e < n) W[e] = nan;
    if (V && e < (int64_t)n * n) V[(e / n) * ldv + e % n] = nan;
}

// The merge tree: halves until single entries; merges grouped by height so
// each level's merges are disjoint and their halves are done.
struct DcPlan {
    std::vector<int4> merges;   // level by level
    std::vector<int> level_off;  // merges[level_off[l], level_off[l+1])
    std::vector<int> level_mmax;
    std::vector<unsigned char> split;
};

int dc_tree(int lo, int hi, std::vector<std::vector<int4>> &by_h) {
    if (hi - lo <= 1) return 0;
    const int mid = lo + (hi - lo) / 2;
    const int h = 1 + std::max(dc_tree(lo, mid, by_h), dc_tree(mid, hi, by_h));
    if ((int)by_h.size() < h) by_h.resize(h);
    by_h[h - 1].push_back(make_int4(lo, mid, hi, 0));
    return h;
}

DcPlan dc_plan(int n) {
    DcPlan p;
    std::vector<std::vector<int4>> by_h;
    dc_tree(0, n, by_h);
    p.split.assign((size_t)n + 1, 0);
    p.level_off.push_back(0);
    for (auto &lv : by_h) {
        int mm = 0;
        for (const int4 &m : lv) {
            p.merges.push_back(m);
            p.split[m.y] = 1;
            mm = std::max(mm, m.z - m.x);
        }
        p.level_off.push_back((int)p.merges.size());
        p.level_mmax.push_back(mm);
    }
    return p;
}

// Merges at or below this size multiply in one CTA; above it, on the GEMM.
constexpr int kDcSmallMerge = 64;

template <typename T>
int syevd(nmx_ctx ctx, int64_t n64, const T *A, int64_t lda, T *W, T *V, int64_t ldv,
          int32_t *info, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(n64 >= 0 && n64 <= (int64_t(1) << 20), 2, "n out of range");
    NMX_ARG_CHECK(A != nullptr || n64 == 0, 3, "A is NULL");
    NMX_ARG_CHECK(lda >= std::max<int64_t>(1, n64), 4, "lda < max(1, n)");
    NMX_ARG_CHECK(W != nullptr || n64 == 0, 5, "W is NULL");
    NMX_ARG_CHECK(V == nullptr || ldv >= std::max<int64_t>(1, n64), 7, "ldv < max(1, n)");
    NMX_ARG_CHECK(info != nullptr, 8, "info is NULL");
    const int n = (int)n64;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    NMX_CUDA_TRY(cudaMemsetAsync(info, 0, sizeof(int32_t), st));
    if (n == 0) return 0;

    // Cooperative grid of the tridiagonalization: one CTA per SM.
    int per_sm = 0;
    NMX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, latrd_kernel, kTrdThreads, 0));
    const int G = std::min(ctx->sm_count, std::max(per_sm, 0) * ctx->sm_count);
    if (G < 1 || (int64_t)(n - 1) > (int64_t)kTrdRows * G * kTrdWarps) {
        set_error("eigh: order %d exceeds the cooperative tridiagonalization's %d rows", n,
                  kTrdRows * std::max(G, 0) * kTrdWarps + 1);
        return NMX_ERR_UNSUPPORTED;
    }
    const bool vectors = V != nullptr;
    const DcPlan plan = vectors ? dc_plan(n) : DcPlan{};
    int mmax = 1;
    for (int m : plan.level_mmax) mmax = std::max(mmax, m);
    const size_t nn = (size_t)n * n, nm = (size_t)n * mmax;
    // Work copy, vectors and scalars; then the divide and conquer's buffers.
    size_t doubles = nn + 5 * (size_t)n + 2 * (size_t)kLrdNb * n + 2 * (size_t)kLrdVec * G + 64;
    if (vectors)
        doubles += nn + 3 * nm + 12 * (size_t)n + plan.merges.size() * 2 + 16;
    size_t ints = 8 * (size_t)n + 3 * plan.merges.size() + 64;
    const size_t bytes = sizeof(double) * doubles + sizeof(int) * ints +
                         sizeof(int4) * plan.merges.size() + (size_t)n + 1024;
    void *wsv = nullptr;
    NMX_TRY(ctx->ensure_slot(kWsEig, bytes, &wsv));
    double *ws = static_cast<double *>(wsv);
    double *Aw = ws;
    double *d = Aw + nn, *e = d + n, *tau = e + n, *xbuf = tau + n, *ybuf = xbuf + n;
    double *Vp = ybuf + n, *Wp = Vp + (size_t)kLrdNb * n;
    double *part = Wp + (size_t)kLrdNb * n;
    double *cur = part + 2 * (size_t)kLrdVec * G;
    DcBuf b{};
    if (vectors) {
        b.Qa = cur;
        b.Qsel = b.Qa + nn;
        b.Ut = b.Qsel + nm;
        b.Qout = b.Ut + nm;
        double *v = b.Qout + nm;
        b.D = v;
        b.e = v + n;
        b.zvec = v + 2 * (size_t)n;
        b.ds = v + 3 * (size_t)n;
        b.zs = v + 4 * (size_t)n;
        b.dl = v + 5 * (size_t)n;
        b.zl = v + 6 * (size_t)n;
        b.ddef = v + 7 * (size_t)n;
        b.rc = v + 8 * (size_t)n;
        b.rs = v + 9 * (size_t)n;
        b.tau = v + 10 * (size_t)n;
        b.zhat = v + 11 * (size_t)n;
        b.rho = v + 12 * (size_t)n;
        b.norm = b.rho + plan.merges.size();
        cur = b.norm + 16;
    }
    cur += 8;
    unsigned long long *maxabs = reinterpret_cast<unsigned long long *>(cur);
    unsigned *bar = reinterpret_cast<unsigned *>(maxabs + 1);
    int *ip = reinterpret_cast<int *>(bar + 2);
    int *err = ip;
    int *scale_exp = ip + 1;
    ip += 8;
    if (vectors) {
        b.perm = ip;
        b.cnd = ip + n;
        b.cdef = ip + 2 * (size_t)n;
        b.ra = ip + 3 * (size_t)n;
        b.rb = ip + 4 * (size_t)n;
        b.org = ip + 5 * (size_t)n;
        b.slot = ip + 6 * (size_t)n;
        b.kc = ip + 7 * (size_t)n;
        ip = b.kc + 3 * plan.merges.size();
    }
    int4 *mg_dev = reinterpret_cast<int4 *>(((uintptr_t)ip + 15) & ~uintptr_t(15));
    unsigned char *split_dev = reinterpret_cast<unsigned char *>(mg_dev + plan.merges.size());

    // 1. symmetric FP64 work copy and max |a|.
    NMX_CUDA_TRY(cudaMemsetAsync(maxabs, 0, sizeof(unsigned long long) + 2 * sizeof(unsigned) +
                                                8 * sizeof(int),
                                 st));
    const unsigned tiles = (unsigned)ceil_div(n, 32);
    sym_lower_kernel<T><<<dim3(tiles, tiles), 256, 0, st>>>(A, lda, n, Aw, n, maxabs);
    NMX_CUDA_TRY(cudaGetLastError());
    // A NaN or an infinity anywhere in the lower triangle ends the call here.
    unsigned long long amax_bits = 0;
    NMX_CUDA_TRY(cudaMemcpyAsync(&amax_bits, maxabs, sizeof(amax_bits), cudaMemcpyDeviceToHost, st));
    NMX_CUDA_TRY(cudaStreamSynchronize(st));
    double amax = 0.0;
    std::memcpy(&amax, &amax_bits, sizeof(amax));
    if (!(amax <= 1.7976931348623157e308)) {
        nonfinite_kernel<T><<<(unsigned)ceil_div((int64_t)n * (V ? n : 1), 256), 256, 0, st>>>(
            n, W, V, ldv, info);
        NMX_CUDA_TRY(cudaGetLastError());
        NMX_CUDA_TRY(cudaStreamSynchronize(st));
        return 0;
    }

    // 2. tridiagonalization: an exact power-of-two scale, then the panels.
    int ex = 0;
    if (amax > 0.0) std::frexp(amax, &ex);
    NMX_CUDA_TRY(cudaMemcpyAsync(scale_exp, &ex, sizeof(int), cudaMemcpyHostToDevice, st));
    if (ex != 0) {
        scale_kernel<<<(unsigned)ceil_div((int64_t)n * n, 256), 256, 0, st>>>(Aw, (int64_t)n * n, ex);
        NMX_CUDA_TRY(cudaGetLastError());
    }
    for (int p = 0; p + 2 < n; p += kLrdNb) {
        const int jb = std::min(kLrdNb, n - 2 - p);
        NMX_CUDA_TRY(cudaMemsetAsync(bar, 0, sizeof(unsigned), st));
        LrdArgs la{Aw, (int64_t)n, n, p, jb, d, e, tau, Vp, Wp, xbuf, ybuf, part, bar, err};
        void *args[] = {&la};
        NMX_CUDA_TRY(cudaLaunchCooperativeKernel((void *)latrd_kernel, dim3(G), dim3(kTrdThreads),
                                                 args, 0, st));
        const int q = p + jb, M = n - q;
        const size_t off = (size_t)q * kLrdNb;
        double *C = Aw + (size_t)q * n + q;
        NMX_TRY(gemm_cc<double>(st, false, true, M, M, jb, -1.0, Vp + off, kLrdNb, Wp + off, kLrdNb,
                                1.0, C, n));
        NMX_TRY(gemm_cc<double>(st, false, true, M, M, jb, -1.0, Wp + off, kLrdNb, Vp + off, kLrdNb,
                                1.0, C, n));
    }
    trd_tail_kernel<<<1, 32, 0, st>>>(Aw, n, n, d, e, tau);
    NMX_CUDA_TRY(cudaGetLastError());

    if (!vectors) {
        // One thread per eigenvalue in 32-thread CTAs: every SM gets work.
        bisect_kernel<T><<<(unsigned)ceil_div(n, 32), 32, 0, st>>>(n, d, e, scale_exp, W);
        NMX_CUDA_TRY(cudaGetLastError());
    } else {
        // 3. divide and conquer.
        NMX_CUDA_TRY(cudaMemcpyAsync(mg_dev, plan.merges.data(), sizeof(int4) * plan.merges.size(),
                                     cudaMemcpyHostToDevice, st));
        NMX_CUDA_TRY(cudaMemcpyAsync(split_dev, plan.split.data(), (size_t)n,
                                     cudaMemcpyHostToDevice, st));
        dc_norm_kernel<<<1, 1024, 0, st>>>(n, d, e, b.norm);
        dc_init_kernel<<<(unsigned)ceil_div((int64_t)n * n, 256), 256, 0, st>>>(
            n, d, e, split_dev, b.norm, b.D, b.e, b.Qa);
        NMX_CUDA_TRY(cudaGetLastError());
        std::vector<int> kc;
        for (size_t l = 0; l + 1 < plan.level_off.size(); ++l) {
            const int off = plan.level_off[l], cnt = plan.level_off[l + 1] - off;
            const int mm = plan.level_mmax[l];
            const int4 *mgl = mg_dev + off;
            DcBuf bl = b;
            bl.rho = b.rho + off;
            bl.kc = b.kc + 3 * off;
            dc_deflate_kernel<<<cnt, 128, 0, st>>>(mgl, n, bl);
            dc_rotate_kernel<<<dim3((unsigned)ceil_div(mm, 8), cnt), 256, 0, st>>>(mgl, n, bl);
            // One thread per root (per z-hat entry) in 32-thread CTAs, so
            // the top levels' few merges still spread over every SM.
            dc_secular_kernel<<<dim3((unsigned)ceil_div(mm, 32), cnt), 32, 0, st>>>(mgl, bl);
            dc_zhat_kernel<<<dim3((unsigned)ceil_div(mm, 32), cnt), 32, 0, st>>>(mgl, bl);
            dc_vec_kernel<<<dim3(mm, cnt), 128, 0, st>>>(mgl, mmax, bl);
            dc_gather_kernel<<<dim3((unsigned)ceil_div((int64_t)mm * mm, 256), cnt), 256, 0, st>>>(
                mgl, n, mmax, bl);
            NMX_CUDA_TRY(cudaGetLastError());
            if (mm <= kDcSmallMerge) {
                dc_small_gemm_kernel<<<cnt, 256, 0, st>>>(mgl, mmax, bl);
            } else {
                // The GEMM sizes need each merge's surviving count.
                kc.resize((size_t)3 * cnt);
                NMX_CUDA_TRY(cudaMemcpyAsync(kc.data(), bl.kc, sizeof(int) * 3 * cnt,
                                             cudaMemcpyDeviceToHost, st));
                NMX_CUDA_TRY(cudaStreamSynchronize(st));
                for (int q = 0; q < cnt; ++q) {
                    const int4 m4 = plan.merges[off + q];
                    const int m = m4.z - m4.x, k = kc[3 * q];
                    if (k == 0) continue;
                    const size_t o = (size_t)m4.x * mmax;
                    NMX_TRY(gemm_cc<double>(st, false, true, m, k, k, 1.0, b.Qsel + o, m, b.Ut + o,
                                            k, 0.0, b.Qout + o, k));
                }
            }
            dc_rank_kernel<<<dim3((unsigned)ceil_div(mm, 128), cnt), 128, 0, st>>>(mgl, bl);
            dc_write_kernel<<<dim3((unsigned)ceil_div(mm, 8), cnt), 256, 0, st>>>(mgl, n, mmax, bl);
            NMX_CUDA_TRY(cudaGetLastError());
        }
        dc_finish_kernel<T><<<(unsigned)ceil_div(n, 256), 256, 0, st>>>(n, b.D, b.norm, scale_exp, W);
        NMX_CUDA_TRY(cudaGetLastError());
        // 4. eigenvectors of A: Q Z, Q's reflectors below Aw's subdiagonal.
        if (n >= 3)
            NMX_TRY(qr_apply_q_f64(ctx, st, n - 1, n - 2, Aw + n, n, tau, b.Qa + n, n, n));
        copy_out_kernel<T><<<(unsigned)ceil_div((int64_t)n * n, 256), 256, 0, st>>>(b.Qa, n, V,
                                                                                  ldv);
        NMX_CUDA_TRY(cudaGetLastError());
    }
    // The barrier's error word: a grid round that gave up.
    int herr = 0;
    NMX_CUDA_TRY(cudaMemcpyAsync(&herr, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    NMX_CUDA_TRY(cudaStreamSynchronize(st));
    if (herr) {
        set_error("eigh: a grid round of the tridiagonalization timed out");
        return NMX_ERR_INTERNAL;
    }
    return 0;
}

}  // namespace
}  // namespace nmx

extern "C" {

NMX_API int nmx_syevd_f64(nmx_ctx ctx, int64_t n, const double *A, int64_t lda, double *W,
                          double *V, int64_t ldv, int32_t *info, void *stream) {
    return nmx::syevd<double>(ctx, n, A, lda, W, V, ldv, info, stream);
}

NMX_API int nmx_syevd_f32(nmx_ctx ctx, int64_t n, const float *A, int64_t lda, float *W, float *V,
                          int64_t ldv, int32_t *info, void *stream) {
    return nmx::syevd<float>(ctx, n, A, lda, W, V, ldv, info, stream);
}

}  // extern "C"
