// Hand-written FP64 (DMMA) and FP32 (FFMA) GEMMs for the dense
// factorizations' updates; interface and scope in gemm_cc.cuh.
//
// One CTA computes a BM x BN tile of C.  Operand tiles of BK columns of the
// inner dimension move from HBM/L2 to shared memory with cp.async (8-byte
// copies for FP64, 4-byte for FP32, so any leading dimension and offset
// works; out-of-range elements are zero-filled), STAGES deep, always stored
// K-major: As[k][m], Bs[k][n], whatever op(A) / op(B) is.
//
// FP64: each warp owns a (BM/WM) x (BN/WN) block of C as 8 x 8 DMMA tiles
// (mma.sync.aligned.m8n8k4.row.col.f64).  Fragment of A: lane l holds
// A[row l/4][k l%4]; of B: B[k l%4][col l/4]; of C: C[row l/4][cols 2(l%4)+0,1].
// A row pitch of BM+4 (BN+4) doubles puts the 16 lanes of a half-warp --
// 4 k's x 4 rows -- on 16 different 8-byte bank pairs: conflict-free.
//
// FP32: 256 threads as a 16 x 16 grid; thread (ty, tx) accumulates the rows
// {4ty..4ty+3, BM/2+4ty..} x columns {4tx.., BN/2+4tx..} (two 4x4 halves so
// that a warp's float4 reads of Bs are contiguous and its reads of As are
// broadcasts), 64 (or 16) FFMA per k per thread.
#include <algorithm>

#include "gemm_cc.cuh"
#include "nmx_common.cuh"

namespace nmx {

namespace {

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}
// src_bytes == 0 zero-fills the destination without reading src.
__device__ __forceinline__ void cp_async8(unsigned dst, const void *src, bool pred) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(dst), "l"(src),
                 "r"(pred ? 8 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_async4(unsigned dst, const void *src, bool pred) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(dst), "l"(src),
                 "r"(pred ? 4 : 0)
                 : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory");
}

template <typename T>
struct GemmArgs {
    int64_t m, n, k;
    T alpha, beta;
    const T *A;
    int64_t lda;
    const T *B;
    int64_t ldb;
    T *C;
    int64_t ldc;
    int lower;
};

// Copy the BK-deep slice at k0 of op(A) (rows m0..m0+BM) and op(B) (columns
// n0..n0+BN) into the stage's K-major tiles.  Element (m, k) of op(A) is
// A[m lda + k] (TA false) or A[k lda + m]; (k, n) of op(B) is B[k ldb + n]
// (TB false) or B[n ldb + k].  Thread order follows the contiguous index so
// that global reads coalesce.
// Shared-memory placement of a tile: K-major ([k][m], pitch BM + 4) or
// M-major ([m][k], pitch BK + 4).  The FP64 kernel keeps each operand in the
// order its rows arrive from memory (row-major A: M-major; B^T: N-major), so
// the copies land on consecutive addresses and the fragment reads stay
// conflict-free either way; the FP32 kernel reads K-major tiles as float4.
template <int BM, int BK, bool MMAJOR>
__device__ __forceinline__ int tile_index(int mm, int kk) {
    return MMAJOR ? mm * (BK + 4) + kk : kk * (BM + 4) + mm;
}
template <int BM, int BK, bool MMAJOR>
__host__ __device__ constexpr int tile_elems() {
    return MMAJOR ? BM * (BK + 4) : BK * (BM + 4);
}

template <typename T, int BM, int BN, int BK, int NT, bool TA, bool TB, bool AM = false,
          bool BN_MAJOR = false>
__device__ __forceinline__ void load_stage(const GemmArgs<T> &p, int64_t m0, int64_t n0,
                                           int64_t k0, T *As, T *Bs) {
    const int tid = threadIdx.x;
#pragma unroll
    for (int e = tid; e < BM * BK; e += NT) {
        int mm, kk;
        if (TA) {
            kk = e / BM;
            mm = e % BM;
        } else {
            mm = e / BK;
            kk = e % BK;
        }
        const int64_t gm = m0 + mm, gk = k0 + kk;
        const bool ok = gm < p.m && gk < p.k;
        const T *src = ok ? (TA ? p.A + gk * p.lda + gm : p.A + gm * p.lda + gk) : p.A;
        const int si = tile_index<BM, BK, AM>(mm, kk);
        if (sizeof(T) == 8)
            cp_async8(smem_u32(As + si), src, ok);
        else
            cp_async4(smem_u32(As + si), src, ok);
    }
#pragma unroll
    for (int e = tid; e < BN * BK; e += NT) {
        int nn, kk;
        if (TB) {
            nn = e / BK;
            kk = e % BK;
        } else {
            kk = e / BN;
            nn = e % BN;
        }
        const int64_t gn = n0 + nn, gk = k0 + kk;
        const bool ok = gn < p.n && gk < p.k;
        const T *src = ok ? (TB ? p.B + gn * p.ldb + gk : p.B + gk * p.ldb + gn) : p.B;
        const int si = tile_index<BN, BK, BN_MAJOR>(nn, kk);
        if (sizeof(T) == 8)
            cp_async8(smem_u32(Bs + si), src, ok);
        else
            cp_async4(smem_u32(Bs + si), src, ok);
    }
}

// The epilogue of one thread: R rows of C, each with one run of W
// consecutive columns (c0[i], c0[i] + W), holding acc[i][0..W).  Every C
// value is loaded before any is stored: a store may alias a later load, so
// interleaving them would make each load wait for the previous store's load
// to return.  Runs of two use 16-byte accesses when C and ldc allow.
template <typename T, int R, int W>
__device__ __forceinline__ void epilogue(const GemmArgs<T> &p, const int64_t (&r)[R],
                                         const int64_t (&c0)[R], T (&acc)[R][W]) {
    const bool pair_ok = W == 2 && sizeof(T) == 8 &&
                         ((reinterpret_cast<uintptr_t>(p.C) & 15) == 0) && ((p.ldc & 1) == 0);
    if (p.beta != T(0)) {
        T old[R][W];
#pragma unroll
        for (int i = 0; i < R; ++i) {
            const T *src = p.C + r[i] * p.ldc + c0[i];
            const bool row_ok = r[i] < p.m;
            if (pair_ok && row_ok && c0[i] + 1 < p.n) {
                const double2 v = *reinterpret_cast<const double2 *>(src);
                old[i][0] = (T)v.x;
                old[i][W - 1] = (T)v.y;
            } else {
#pragma unroll
                for (int j = 0; j < W; ++j)
                    old[i][j] = (row_ok && c0[i] + j < p.n) ? src[j] : T(0);
            }
        }
#pragma unroll
        for (int i = 0; i < R; ++i)
#pragma unroll
            for (int j = 0; j < W; ++j) acc[i][j] = p.alpha * acc[i][j] + p.beta * old[i][j];
    } else {
#pragma unroll
        for (int i = 0; i < R; ++i)
#pragma unroll
            for (int j = 0; j < W; ++j) acc[i][j] = p.alpha * acc[i][j];
    }
#pragma unroll
    for (int i = 0; i < R; ++i) {
        if (r[i] >= p.m) continue;
        T *dst = p.C + r[i] * p.ldc + c0[i];
        const bool full = c0[i] + W - 1 < p.n && (!p.lower || c0[i] + W - 1 <= r[i]);
        if (pair_ok && full) {
            *reinterpret_cast<double2 *>(dst) = make_double2((double)acc[i][0], (double)acc[i][W - 1]);
        } else {
#pragma unroll
            for (int j = 0; j < W; ++j)
                if (c0[i] + j < p.n && (!p.lower || c0[i] + j <= r[i])) dst[j] = acc[i][j];
        }
    }
}

// Tiles entirely above C's diagonal do nothing in the lower-triangle mode.
template <int BM, int BN>
__device__ __forceinline__ bool tile_skipped(int lower, int64_t m0, int64_t n0) {
    return lower && n0 > m0 + BM - 1;
}

// ---- FP64: DMMA ---------------------------------------------------------

// KS > 1 splits each 16-deep slice of K over KS groups of WM x WN warps
// (group g takes the k4 steps g, g + KS, ...) and sums the groups' partial
// tiles through shared memory at the end, in group order: more warps for the
// tiles of a thin product (few columns, long K) without a second pass.
template <int BM, int BN, int WM, int WN, bool TA, bool TB, int KS = 1>
__global__ void __launch_bounds__(WM *WN * 32 * KS) dgemm_kernel(GemmArgs<double> p) {
    constexpr int BK = 16, STAGES = 3, NT = WM * WN * 32 * KS;
    constexpr bool AM = !TA, BNM = TB;  // M-major A, N-major B (see tile_index)
    constexpr int SA = tile_elems<BM, BK, AM>(), SB = tile_elems<BN, BK, BNM>();
    constexpr int TM = BM / WM, TN = BN / WN, FM = TM / 8, FN = TN / 8;
    static_assert(KS == 1 || KS == 2 || KS == 4, "K split of 1, 2 or 4 groups");
    extern __shared__ __align__(16) double dsm[];
    double *As = dsm;
    double *Bs = dsm + STAGES * SA;
    const int64_t m0 = (int64_t)blockIdx.y * BM, n0 = (int64_t)blockIdx.x * BN;
    if (tile_skipped<BM, BN>(p.lower, m0, n0)) return;
    const int warp_all = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ks = warp_all / (WM * WN), warp = warp_all % (WM * WN);
    const int wm0 = (warp / WN) * TM, wn0 = (warp % WN) * TN;
    const int fr = lane >> 2, fk = lane & 3;
    double acc[FM][FN][2];
#pragma unroll
    for (int i = 0; i < FM; ++i)
#pragma unroll
        for (int j = 0; j < FN; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
    const int KT = (int)ceil_div(p.k, BK);
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < KT)
            load_stage<double, BM, BN, BK, NT, TA, TB, AM, BNM>(p, m0, n0, (int64_t)s * BK,
                                                               As + s * SA, Bs + s * SB);
        cp_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        cp_wait<STAGES - 2>();
        __syncthreads();
        {
            const int nk = kt + STAGES - 1, s = nk % STAGES;
            if (nk < KT)
                load_stage<double, BM, BN, BK, NT, TA, TB, AM, BNM>(p, m0, n0, (int64_t)nk * BK,
                                                                   As + s * SA, Bs + s * SB);
            cp_commit();
        }
        const double *as = As + (kt % STAGES) * SA;
        const double *bs = Bs + (kt % STAGES) * SB;
#pragma unroll
        for (int k4 = 4 * ks; k4 < BK; k4 += 4 * KS) {
            double a[FM], b[FN];
#pragma unroll
            for (int i = 0; i < FM; ++i) a[i] = as[tile_index<BM, BK, AM>(wm0 + i * 8 + fr, k4 + fk)];
#pragma unroll
            for (int j = 0; j < FN; ++j) b[j] = bs[tile_index<BN, BK, BNM>(wn0 + j * 8 + fr, k4 + fk)];
#pragma unroll
            for (int i = 0; i < FM; ++i)
#pragma unroll
                for (int j = 0; j < FN; ++j)
                    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, "
                        "{%0,%1};\n"
                        : "+d"(acc[i][j][0]), "+d"(acc[i][j][1])
                        : "d"(a[i]), "d"(b[j]));
        }
    }
    cp_wait<0>();
    if constexpr (KS > 1) {
        // Groups 1.. leave their partial tiles in shared memory (the pipeline
        // buffers are free now); group 0 adds them in group order.
        __syncthreads();
        double *red = dsm;
        constexpr int per = FM * FN * 2 * 32;  // doubles per warp
        if (ks > 0) {
#pragma unroll
            for (int i = 0; i < FM; ++i)
#pragma unroll
                for (int j = 0; j < FN; ++j)
#pragma unroll
                    for (int e = 0; e < 2; ++e)
                        red[((ks - 1) * WM * WN + warp) * per + ((i * FN + j) * 2 + e) * 32 + lane] =
                            acc[i][j][e];
        }
        __syncthreads();
        if (ks > 0) return;
#pragma unroll
        for (int g = 1; g < KS; ++g)
#pragma unroll
            for (int i = 0; i < FM; ++i)
#pragma unroll
                for (int j = 0; j < FN; ++j)
#pragma unroll
                    for (int e = 0; e < 2; ++e)
                        acc[i][j][e] += red[((g - 1) * WM * WN + warp) * per +
                                            ((i * FN + j) * 2 + e) * 32 + lane];
    }
    // Epilogue in groups of FN tiles: row i of every group's tiles.
#pragma unroll
    for (int i = 0; i < FM; ++i) {
        int64_t r[FN], c0[FN];
#pragma unroll
        for (int j = 0; j < FN; ++j) {
            r[j] = m0 + wm0 + i * 8 + fr;
            c0[j] = n0 + wn0 + j * 8 + 2 * fk;
        }
        epilogue<double, FN, 2>(p, r, c0, acc[i]);
    }
}

// ---- FP32: FFMA ---------------------------------------------------------

// R consecutive floats of shared memory (R = 2 or a multiple of 4; the
// address is aligned to 4R bytes up to 16).
template <int R>
__device__ __forceinline__ void load_run(const float *src, float *dst) {
    if constexpr (R % 4 == 0) {
#pragma unroll
        for (int q = 0; q < R; q += 4) {
            const float4 v = *reinterpret_cast<const float4 *>(src + q);
            dst[q] = v.x;
            dst[q + 1] = v.y;
            dst[q + 2] = v.z;
            dst[q + 3] = v.w;
        }
    } else {
        static_assert(R == 2, "micro-tile runs are 2 or multiples of 4");
        const float2 v = *reinterpret_cast<const float2 *>(src);
        dst[0] = v.x;
        dst[1] = v.y;
    }
}

// 256 threads; micro-tile (BM/16) x (BN/16) per thread as two halves.
template <int BM, int BN, bool TA, bool TB>
__global__ void __launch_bounds__(256) sgemm_kernel(GemmArgs<float> p) {
    constexpr int BK = 8, STAGES = 4, NT = 256;
    constexpr int PA = BM + 4, PB = BN + 4;
    constexpr int RM = BM / 32, RN = BN / 32;  // rows / columns per half per thread
    extern __shared__ __align__(16) float fsm[];
    float *As = fsm;
    float *Bs = fsm + STAGES * BK * PA;
    const int64_t m0 = (int64_t)blockIdx.y * BM, n0 = (int64_t)blockIdx.x * BN;
    if (tile_skipped<BM, BN>(p.lower, m0, n0)) return;
    const int ty = threadIdx.x >> 4, tx = threadIdx.x & 15;
    float acc[2 * RM][2 * RN];
#pragma unroll
    for (int i = 0; i < 2 * RM; ++i)
#pragma unroll
        for (int j = 0; j < 2 * RN; ++j) acc[i][j] = 0.f;
    const int KT = (int)ceil_div(p.k, BK);
#pragma unroll
    for (int s = 0; s < STAGES - 1; ++s) {
        if (s < KT)
            load_stage<float, BM, BN, BK, NT, TA, TB>(p, m0, n0, (int64_t)s * BK, As + s * BK * PA,
                                                     Bs + s * BK * PB);
        cp_commit();
    }
    for (int kt = 0; kt < KT; ++kt) {
        cp_wait<STAGES - 2>();
        __syncthreads();
        {
            const int nk = kt + STAGES - 1, s = nk % STAGES;
            if (nk < KT)
                load_stage<float, BM, BN, BK, NT, TA, TB>(p, m0, n0, (int64_t)nk * BK,
                                                         As + s * BK * PA, Bs + s * BK * PB);
            cp_commit();
        }
        const float *as = As + (kt % STAGES) * BK * PA;
        const float *bs = Bs + (kt % STAGES) * BK * PB;
#pragma unroll
        for (int kk = 0; kk < BK; ++kk) {
            float a[2 * RM], b[2 * RN];
#pragma unroll
            for (int h = 0; h < 2; ++h) {
                load_run<RM>(as + kk * PA + h * (BM / 2) + ty * RM, a + h * RM);
                load_run<RN>(bs + kk * PB + h * (BN / 2) + tx * RN, b + h * RN);
            }
#pragma unroll
            for (int i = 0; i < 2 * RM; ++i)
#pragma unroll
                for (int j = 0; j < 2 * RN; ++j) acc[i][j] = fmaf(a[i], b[j], acc[i][j]);
        }
    }
    cp_wait<0>();
    // Epilogue per row of the micro-tile: its two column runs of RN.
#pragma unroll
    for (int i = 0; i < 2 * RM; ++i) {
        int64_t r[2], c0[2];
        float v[2][RN];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            r[h] = m0 + (i / RM) * (BM / 2) + ty * RM + (i % RM);
            c0[h] = n0 + h * (BN / 2) + tx * RN;
#pragma unroll
            for (int q = 0; q < RN; ++q) v[h][q] = acc[i][h * RN + q];
        }
        epilogue<float, 2, RN>(p, r, c0, v);
    }
}

// ---- launch ---------------------------------------------------------------

template <int BM, int BN, int WM, int WN, bool TA, bool TB, int KS = 1>
int launch_d(cudaStream_t st, const GemmArgs<double> &p) {
    constexpr int BK = 16, STAGES = 3;
    constexpr size_t pipe =
        sizeof(double) * STAGES * (tile_elems<BM, BK, !TA>() + tile_elems<BN, BK, TB>());
    constexpr size_t red = sizeof(double) * (KS - 1) * BM * BN;
    const size_t smem = pipe > red ? pipe : red;
    auto kern = dgemm_kernel<BM, BN, WM, WN, TA, TB, KS>;
    static bool attr[64] = {};
    int dev = 0;
    NMX_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        NMX_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr[dev] = true;
    }
    dim3 grid((unsigned)ceil_div(p.n, BN), (unsigned)ceil_div(p.m, BM));
    kern<<<grid, WM * WN * 32 * KS, smem, st>>>(p);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

template <int BM, int BN, bool TA, bool TB>
int launch_s(cudaStream_t st, const GemmArgs<float> &p) {
    constexpr int BK = 8, STAGES = 4;
    const size_t smem = sizeof(float) * STAGES * BK * ((BM + 4) + (BN + 4));
    auto kern = sgemm_kernel<BM, BN, TA, TB>;
    static bool attr[64] = {};
    int dev = 0;
    NMX_CUDA_TRY(cudaGetDevice(&dev));
    if (dev < 64 && !attr[dev]) {
        NMX_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        attr[dev] = true;
    }
    dim3 grid((unsigned)ceil_div(p.n, BN), (unsigned)ceil_div(p.m, BM));
    kern<<<grid, 256, smem, st>>>(p);
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

inline bool big_tiles(const GemmArgs<float> &p, int sms) {
    return ceil_div(p.m, 128) * ceil_div(p.n, 128) >= (int64_t)sms;
}

// FP64 tile by shape, from a sweep of tile shapes over the factorizations'
// products on B200 (DMMA at 128 FLOP/clk/SM): 32 x 16 tiles with a 4-way K
// split for products of <= 32 columns (the solves' right-hand sides, the
// recursion's narrowest panels), 64 x 64 for the K = 256 look-ahead updates
// and other thin-K or narrow products, 64 x 128 for the rest (long K,
// 128..256 columns).
template <bool TA, bool TB>
int dispatch(cudaStream_t st, const GemmArgs<double> &p, int) {
    if (p.n <= 32) return launch_d<32, 16, 2, 1, TA, TB, 4>(st, p);
    if (p.n <= 64 || (p.n > 256 && p.k < 1024)) return launch_d<64, 64, 2, 2, TA, TB>(st, p);
    return launch_d<64, 128, 2, 2, TA, TB>(st, p);
}
template <bool TA, bool TB>
int dispatch(cudaStream_t st, const GemmArgs<float> &p, int sms) {
    if (big_tiles(p, sms)) return launch_s<128, 128, TA, TB>(st, p);
    return launch_s<64, 64, TA, TB>(st, p);
}

int device_sms() {
    static int sms[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return 148;
    if (!sms[dev]) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || v <= 0)
            v = 148;
        sms[dev] = v;
    }
    return sms[dev];
}

}  // namespace

template <typename T>
int gemm_cc(cudaStream_t st, bool ta, bool tb, int64_t m, int64_t n, int64_t k, T alpha,
            const T *A, int64_t lda, const T *B, int64_t ldb, T beta, T *C, int64_t ldc,
            bool lower) {
    if (m <= 0 || n <= 0) return 0;
    if (ceil_div(m, 64) > 65535) {
        set_error("gemm: %lld rows exceed the grid limit", (long long)m);
        return NMX_ERR_UNSUPPORTED;
    }
    GemmArgs<T> p{m, n, std::max<int64_t>(k, 0), alpha, beta, A, lda, B, ldb, C, ldc, lower ? 1 : 0};
    if (k <= 0) {  // C = beta C: the K loop is empty, the epilogue scales.
        p.k = 0;
    }
    const int sms = device_sms();
    if (!ta && !tb) return dispatch<false, false>(st, p, sms);
    if (!ta && tb) return dispatch<false, true>(st, p, sms);
    if (ta && !tb) return dispatch<true, false>(st, p, sms);
    return dispatch<true, true>(st, p, sms);
}

template int gemm_cc<double>(cudaStream_t, bool, bool, int64_t, int64_t, int64_t, double,
                             const double *, int64_t, const double *, int64_t, double, double *,
                             int64_t, bool);
template int gemm_cc<float>(cudaStream_t, bool, bool, int64_t, int64_t, int64_t, float,
                            const float *, int64_t, const float *, int64_t, float, float *,
                            int64_t, bool);

}  // namespace nmx

// C-ABI: the general product, for the tests and for callers that want the
// library's own GEMM (numax routes its updates through MAX linalg.matmul,
// numax/linalg/lu.mojo:646-673).
extern "C" NMX_API int nmx_gemm_f64(nmx_ctx ctx, int trans_a, int trans_b, int64_t m, int64_t n,
                                    int64_t k, double alpha, const double *A, int64_t lda,
                                    const double *B, int64_t ldb, double beta, double *C,
                                    int64_t ldc, int lower, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(m >= 0 && n >= 0 && k >= 0, 4, "negative size");
    NMX_ARG_CHECK(lda >= std::max<int64_t>(1, trans_a ? m : k), 9, "lda too small");
    NMX_ARG_CHECK(ldb >= std::max<int64_t>(1, trans_b ? k : n), 11, "ldb too small");
    NMX_ARG_CHECK(ldc >= std::max<int64_t>(1, n), 14, "ldc < n");
    nmx::DeviceGuard g(ctx->device);
    return nmx::gemm_cc<double>(static_cast<cudaStream_t>(stream), trans_a != 0, trans_b != 0, m,
                                n, k, alpha, A, lda, B, ldb, beta, C, ldc, lower != 0);
}
extern "C" NMX_API int nmx_gemm_f32(nmx_ctx ctx, int trans_a, int trans_b, int64_t m, int64_t n,
                                    int64_t k, float alpha, const float *A, int64_t lda,
                                    const float *B, int64_t ldb, float beta, float *C, int64_t ldc,
                                    int lower, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(m >= 0 && n >= 0 && k >= 0, 4, "negative size");
    NMX_ARG_CHECK(lda >= std::max<int64_t>(1, trans_a ? m : k), 9, "lda too small");
    NMX_ARG_CHECK(ldb >= std::max<int64_t>(1, trans_b ? k : n), 11, "ldb too small");
    NMX_ARG_CHECK(ldc >= std::max<int64_t>(1, n), 14, "ldc < n");
    nmx::DeviceGuard g(ctx->device);
    return nmx::gemm_cc<float>(static_cast<cudaStream_t>(stream), trans_a != 0, trans_b != 0, m, n,
                               k, alpha, A, lda, B, ldb, beta, C, ldc, lower != 0);
}
