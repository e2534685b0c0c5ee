// Tensor-core trailing update for the mixed-precision factorizations:
//
//     C[M x N] (fp32, row-major, ldc)  -=  A[M x K] * B[K x N]
//
// with A and B rounded to BF16 or FP16 and the products accumulated in FP32
// on the 5th-generation tensor cores (tcgen05.mma kind::f16, accumulators in
// TMEM, operands staged by TMA) through CUTLASS's sm100 collective builders.
// This is the O(n^3) term of the mixed-precision LU (the role MAX's matmul
// plays in numax/linalg/lu.mojo:646-673, there in fp32 SIMT): the panel and
// the triangular solves stay FP32, only the rank-k update is low precision.
//
// One CTA per 128 x 256 output tile, cluster 1x1x1 (no TMA multicast), fused
// epilogue D = -1 * acc + 1 * C written in place over C.
#include <cutlass/cutlass.h>
#include <cute/tensor.hpp>
#include <cutlass/epilogue/collective/collective_builder.hpp>
#include <cutlass/gemm/collective/collective_builder.hpp>
#include <cutlass/gemm/device/gemm_universal_adapter.h>
#include <cutlass/gemm/dispatch_policy.hpp>
#include <cutlass/gemm/kernel/gemm_universal.hpp>

#include <algorithm>

#include "gemm_tc.cuh"

#pragma nv_diag_suppress 20012

namespace nmx {
namespace tc {

using namespace cute;

// One complete sm100 GEMM type per 16-bit input type, spelled at namespace
// scope (the host compiler rejects the dependent carve-out inside a class
// template).
// LAYOUTB RowMajor: B is K x N with N contiguous (C -= A B); ColumnMajor: B
// is stored N x K with K contiguous (C -= A B^T), its leading dimension the
// stride between its N rows.
#define NMX_TC_GEMM(NAME, ELEM, SCHED, LAYOUTB, BSTRIDE_MODE)                                    \
    namespace NAME {                                                                             \
    using ElementA = ELEM;                                                                       \
    using ElementB = ELEM;                                                                       \
    using LayoutA = cutlass::layout::RowMajor; /* M x K, K contiguous */                         \
    using LayoutB = LAYOUTB;                                                                     \
    using LayoutC = cutlass::layout::RowMajor;                                                   \
    using TileMNK = Shape<_128, _256, _64>;                                                      \
    using ClusterMNK = Shape<_1, _1, _1>;                                                        \
    using Epi = cutlass::epilogue::collective::CollectiveBuilder<                                \
        cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, TileMNK, ClusterMNK,               \
        cutlass::epilogue::collective::EpilogueTileAuto, float, float, float, LayoutC, 4, float, \
        LayoutC, 4, cutlass::epilogue::collective::EpilogueScheduleAuto>::CollectiveOp;          \
    using Main = cutlass::gemm::collective::CollectiveBuilder<                                   \
        cutlass::arch::Sm100, cutlass::arch::OpClassTensorOp, ElementA, LayoutA, 8, ElementB,    \
        LayoutB, 8, float, TileMNK, ClusterMNK,                                                  \
        cutlass::gemm::collective::StageCountAutoCarveout<static_cast<int>(                      \
            sizeof(Epi::SharedStorage))>,                                                        \
        cutlass::gemm::collective::KernelScheduleAuto>::CollectiveOp;                            \
    using Kernel = cutlass::gemm::kernel::GemmUniversal<Shape<int, int, int, int>, Main, Epi,    \
                                                        SCHED>;                                  \
    using Gemm = cutlass::gemm::device::GemmUniversalAdapter<Kernel>;                            \
    inline int run(int M, int N, int K, const void *A, int64_t lda, const void *B, int64_t ldb,  \
                   float *C, int64_t ldc, cudaStream_t st, int sm_count) {                       \
        Kernel::StrideA sa{};                                                                    \
        Kernel::StrideB sb{};                                                                    \
        Kernel::StrideC sc{};                                                                    \
        Kernel::StrideD sd{};                                                                    \
        cute::get<0>(sa) = lda;                                                                  \
        cute::get<BSTRIDE_MODE>(sb) = ldb;                                                       \
        cute::get<0>(sc) = ldc;                                                                  \
        cute::get<0>(sd) = ldc;                                                                  \
        cutlass::KernelHardwareInfo hw;                                                          \
        if (sm_count > 0) {                                                                      \
            cudaGetDevice(&hw.device_id);                                                        \
            hw.sm_count = sm_count;                                                              \
        }                                                                                        \
        Gemm::Arguments args{cutlass::gemm::GemmUniversalMode::kGemm,                            \
                             {M, N, K, 1},                                                       \
                             {static_cast<const ElementA *>(A), sa,                              \
                              static_cast<const ElementB *>(B), sb},                             \
                             {{-1.0f, 1.0f}, C, sc, C, sd},                                      \
                             hw};                                                                \
        Gemm g;                                                                                  \
        if (g.can_implement(args) != cutlass::Status::kSuccess) return 1;                        \
        if (Gemm::get_workspace_size(args) != 0) return 4;                                       \
        if (g.initialize(args, nullptr, st) != cutlass::Status::kSuccess) return 2;              \
        return g.run(st) == cutlass::Status::kSuccess ? 0 : 3;                                   \
    }                                                                                            \
    }

// The default (hardware cluster-launch-control) scheduler takes every SM;
// the static persistent one runs on at most `sm_count` SMs, leaving the rest
// to concurrent work (the look-ahead LU's panel stream).
NMX_TC_GEMM(bf16, cutlass::bfloat16_t, void, cutlass::layout::RowMajor, 1)
NMX_TC_GEMM(fp16, cutlass::half_t, void, cutlass::layout::RowMajor, 1)
NMX_TC_GEMM(bf16s, cutlass::bfloat16_t, cutlass::gemm::StaticPersistentScheduler,
            cutlass::layout::RowMajor, 1)
NMX_TC_GEMM(fp16s, cutlass::half_t, cutlass::gemm::StaticPersistentScheduler,
            cutlass::layout::RowMajor, 1)
// B^T operands (the Cholesky's SYRK and right-side triangular-solve products).
NMX_TC_GEMM(bf16t, cutlass::bfloat16_t, void, cutlass::layout::ColumnMajor, 0)
NMX_TC_GEMM(fp16t, cutlass::half_t, void, cutlass::layout::ColumnMajor, 0)
#undef NMX_TC_GEMM

}  // namespace tc

// fp32 block (rows x cols, ld) -> 16-bit block (rows_p x cols_p, ld_out),
// zero-filled past rows x cols so padded products contribute exactly 0.
template <typename Elem>
__global__ void round_block_kernel(const float *src, int64_t lds, int rows, int cols, int rows_p,
                                   int cols_p, Elem *dst, int64_t ldd) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)rows_p * cols_p) return;
    const int r = (int)(e / cols_p), c = (int)(e - (int64_t)r * cols_p);
    const float v = (r < rows && c < cols) ? src[(int64_t)r * lds + c] : 0.0f;
    dst[(int64_t)r * ldd + c] = Elem(v);
}

// BF16X3 operands: A' = [hi(A) | hi(A) | lo(A)] (rows x 3 cols_p) and
// B' = [hi(B); lo(B); hi(B)] (3 rows_p x cols_p), lo = bf16(x - hi), so one
// GEMM over 3 K gives hi*hi + hi*lo + lo*hi.  Zero past rows x cols.
template <bool IS_A>
__global__ void round_split_bf16_kernel(const float *src, int64_t lds, int rows, int cols,
                                        int rows_p, int cols_p, cutlass::bfloat16_t *dst,
                                        int64_t ldd) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)rows_p * cols_p) return;
    const int r = (int)(e / cols_p), c = (int)(e - (int64_t)r * cols_p);
    const float v = (r < rows && c < cols) ? src[(int64_t)r * lds + c] : 0.0f;
    const cutlass::bfloat16_t hi(v);
    const cutlass::bfloat16_t lo(v - float(hi));
    if (IS_A) {
        cutlass::bfloat16_t *d = dst + (int64_t)r * ldd;
        d[c] = hi;
        d[cols_p + c] = hi;
        d[2 * cols_p + c] = lo;
    } else {
        dst[(int64_t)r * ldd + c] = hi;
        dst[(int64_t)(rows_p + r) * ldd + c] = lo;
        dst[(int64_t)(2 * rows_p + r) * ldd + c] = hi;
    }
}

// BF16X6 operands: x = h + m + l with h = bf16(x), m = bf16(x - h),
// l = bf16(x - h - m) (24 significant bits, FP32's), and the six products
// with i + j <= 2 as one GEMM over 6 K:
//   A' = [h | h | m | h | m | l],  B' = [h; m; h; l; m; h]
// i.e. hh + hm + mh + hl + mm + lh.  The dropped terms are below FP32's
// rounding of the FP32 accumulation.  Zero past rows x cols.
template <bool IS_A>
__global__ void round_split6_bf16_kernel(const float *src, int64_t lds, int rows, int cols,
                                         int rows_p, int cols_p, cutlass::bfloat16_t *dst,
                                         int64_t ldd) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)rows_p * cols_p) return;
    const int r = (int)(e / cols_p), c = (int)(e - (int64_t)r * cols_p);
    const float v = (r < rows && c < cols) ? src[(int64_t)r * lds + c] : 0.0f;
    const cutlass::bfloat16_t h(v);
    const float r1 = v - float(h);
    const cutlass::bfloat16_t m(r1);
    const cutlass::bfloat16_t l(r1 - float(m));
    if (IS_A) {
        cutlass::bfloat16_t *d = dst + (int64_t)r * ldd;
        d[c] = h;
        d[cols_p + c] = h;
        d[2 * cols_p + c] = m;
        d[3 * cols_p + c] = h;
        d[4 * cols_p + c] = m;
        d[5 * cols_p + c] = l;
    } else {
        const cutlass::bfloat16_t seg[6] = {h, m, h, l, m, h};
#pragma unroll
        for (int q = 0; q < 6; ++q) dst[(int64_t)(q * rows_p + r) * ldd + c] = seg[q];
    }
}

static inline int split_factor(int precision) {
    return precision == NMX_PREC_BF16X3 ? 3 : precision == NMX_PREC_BF16X6 ? 6 : 1;
}

// Rows of an fp32 block (rows x cols, lds) rounded or split into 16-bit
// pieces side by side along the row: dst[r][q cols_p + c] = piece number
// (PAT >> 2q) & 3 of src[r][c] (0 = the rounding h, 1 = the residual's
// rounding m, 2 = the second residual's l), for the NSEG segments.  This is
// A's layout for every precision, and B's when B is stored N x K (K-major):
// the segment patterns pair A's pieces with B's, e.g. BF16X3 A = [h h m],
// B = [h m h].  Zero past rows x cols.
template <typename Elem, int NSEG, int PAT>
__global__ void round_rows_kernel(const float *src, int64_t lds, int rows, int cols, int rows_p,
                                  int cols_p, Elem *dst, int64_t ldd) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)rows_p * cols_p) return;
    const int r = (int)(e / cols_p), c = (int)(e - (int64_t)r * cols_p);
    const float v = (r < rows && c < cols) ? src[(int64_t)r * lds + c] : 0.0f;
    Elem piece[3];
    piece[0] = Elem(v);
    if (NSEG > 1) {
        const float r1 = v - float(piece[0]);
        piece[1] = Elem(r1);
        piece[2] = Elem(r1 - float(piece[1]));
    }
    Elem *d = dst + (int64_t)r * ldd;
#pragma unroll
    for (int q = 0; q < NSEG; ++q) d[(int64_t)q * cols_p + c] = piece[(PAT >> (2 * q)) & 3];
}
constexpr int kPatX1 = 0;
constexpr int kPatX3B = (1 << 2);                                   // [h m h]
constexpr int kPatX6B = (1 << 2) | (2 << 6) | (1 << 8);             // [h m h l m h]

// The GEMM runs on K and N rounded up to multiples of 8 (the 16-byte TMA and
// epilogue granularity): the padded rows/columns of the 16-bit operands are
// zero, so the extra columns of C (up to N rounded to 8) get C - 0 and are
// left bit-for-bit unchanged.
static inline int64_t up8(int64_t v) { return (v + 7) / 8 * 8; }

int tc_gemm_sub_f32(cudaStream_t st, int precision, int64_t M, int64_t N, int64_t K, const float *A,
                    int64_t lda, const float *B, int64_t ldb, float *C, int64_t ldc, void *ws,
                    size_t ws_bytes, int sm_limit, bool b_kmajor) {
    if (M <= 0 || N <= 0 || K <= 0) return 0;
    if (b_kmajor) return tc_gemm_sub_bt_f32(st, precision, M, N, K, A, lda, B, ldb, C, ldc, ws, ws_bytes);
    const int64_t Kp = up8(K), Np = up8(N);
    const size_t need = tc_gemm_workspace_bytes(M, N, K, precision);
    if (need > ws_bytes) {
        set_error("tensor-core update needs %zu B of workspace, have %zu", need, ws_bytes);
        return NMX_ERR_INTERNAL;
    }
    if ((ldc % 4) != 0 || (reinterpret_cast<uintptr_t>(C) % 16) != 0 || ldc < Np) {
        set_error("tensor-core update: C must be 16-byte aligned, ldc %% 4 == 0, ldc >= N rounded to 8");
        return NMX_ERR_INTERNAL;
    }
    const int64_t Kw = split_factor(precision) * Kp;  // K of the 16-bit GEMM
    auto *a16 = static_cast<unsigned char *>(ws);
    auto *b16 = a16 + ((2 * (size_t)M * Kw + 255) & ~size_t(255));
    const int threads = 256;
    const unsigned ga = (unsigned)ceil_div(M * Kp, threads), gb = (unsigned)ceil_div(Kp * Np, threads);
    int rc;
    if (precision == NMX_PREC_FP16) {
        auto *a = reinterpret_cast<cutlass::half_t *>(a16);
        auto *b = reinterpret_cast<cutlass::half_t *>(b16);
        round_block_kernel<cutlass::half_t><<<ga, threads, 0, st>>>(A, lda, (int)M, (int)K, (int)M,
                                                                    (int)Kp, a, Kp);
        round_block_kernel<cutlass::half_t><<<gb, threads, 0, st>>>(B, ldb, (int)K, (int)N, (int)Kp,
                                                                    (int)Np, b, Np);
        NMX_CUDA_TRY(cudaGetLastError());
        rc = sm_limit > 0 ? tc::fp16s::run((int)M, (int)Np, (int)Kp, a, Kp, b, Np, C, ldc, st, sm_limit)
                          : tc::fp16::run((int)M, (int)Np, (int)Kp, a, Kp, b, Np, C, ldc, st, 0);
    } else if (precision == NMX_PREC_BF16X3 || precision == NMX_PREC_BF16X6) {
        auto *a = reinterpret_cast<cutlass::bfloat16_t *>(a16);
        auto *b = reinterpret_cast<cutlass::bfloat16_t *>(b16);
        if (precision == NMX_PREC_BF16X3) {
            round_split_bf16_kernel<true><<<ga, threads, 0, st>>>(A, lda, (int)M, (int)K, (int)M,
                                                                  (int)Kp, a, Kw);
            round_split_bf16_kernel<false><<<gb, threads, 0, st>>>(B, ldb, (int)K, (int)N,
                                                                   (int)Kp, (int)Np, b, Np);
        } else {
            round_split6_bf16_kernel<true><<<ga, threads, 0, st>>>(A, lda, (int)M, (int)K, (int)M,
                                                                   (int)Kp, a, Kw);
            round_split6_bf16_kernel<false><<<gb, threads, 0, st>>>(B, ldb, (int)K, (int)N,
                                                                    (int)Kp, (int)Np, b, Np);
        }
        NMX_CUDA_TRY(cudaGetLastError());
        rc = sm_limit > 0 ? tc::bf16s::run((int)M, (int)Np, (int)Kw, a, Kw, b, Np, C, ldc, st, sm_limit)
                          : tc::bf16::run((int)M, (int)Np, (int)Kw, a, Kw, b, Np, C, ldc, st, 0);
    } else {
        auto *a = reinterpret_cast<cutlass::bfloat16_t *>(a16);
        auto *b = reinterpret_cast<cutlass::bfloat16_t *>(b16);
        round_block_kernel<cutlass::bfloat16_t><<<ga, threads, 0, st>>>(A, lda, (int)M, (int)K,
                                                                        (int)M, (int)Kp, a, Kp);
        round_block_kernel<cutlass::bfloat16_t><<<gb, threads, 0, st>>>(B, ldb, (int)K, (int)N,
                                                                        (int)Kp, (int)Np, b, Np);
        NMX_CUDA_TRY(cudaGetLastError());
        rc = sm_limit > 0 ? tc::bf16s::run((int)M, (int)Np, (int)Kp, a, Kp, b, Np, C, ldc, st, sm_limit)
                          : tc::bf16::run((int)M, (int)Np, (int)Kp, a, Kp, b, Np, C, ldc, st, 0);
    }
    if (rc) {
        set_error("tensor-core GEMM %lldx%lldx%lld failed at step %d", (long long)M, (long long)N,
                  (long long)K, rc);
        return NMX_ERR_INTERNAL;
    }
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

// C -= A B^T with B stored N x K (ldb): A rounded / split as in the NN path,
// B rounded / split along its rows (K-major) with the segment pattern that
// pairs with A's, and the K-major-B GEMM.
int tc_gemm_sub_bt_f32(cudaStream_t st, int precision, int64_t M, int64_t N, int64_t K,
                       const float *A, int64_t lda, const float *B, int64_t ldb, float *C,
                       int64_t ldc, void *ws, size_t ws_bytes) {
    if (M <= 0 || N <= 0 || K <= 0) return 0;
    const int64_t Kp = up8(K), Np = up8(N);
    const size_t need = tc_gemm_workspace_bytes(M, N, K, precision);
    if (need > ws_bytes) {
        set_error("tensor-core update needs %zu B of workspace, have %zu", need, ws_bytes);
        return NMX_ERR_INTERNAL;
    }
    if ((ldc % 4) != 0 || (reinterpret_cast<uintptr_t>(C) % 16) != 0 || ldc < Np) {
        set_error("tensor-core update: C must be 16-byte aligned, ldc %% 4 == 0, ldc >= N rounded to 8");
        return NMX_ERR_INTERNAL;
    }
    const int nseg = split_factor(precision);
    const int64_t Kw = nseg * Kp;
    auto *a16 = static_cast<unsigned char *>(ws);
    auto *b16 = a16 + ((2 * (size_t)M * Kw + 255) & ~size_t(255));
    const int threads = 256;
    const unsigned ga = (unsigned)ceil_div(M * Kp, threads), gb = (unsigned)ceil_div(Np * Kp, threads);
    int rc;
    if (precision == NMX_PREC_FP16) {
        auto *a = reinterpret_cast<cutlass::half_t *>(a16);
        auto *b = reinterpret_cast<cutlass::half_t *>(b16);
        round_block_kernel<cutlass::half_t><<<ga, threads, 0, st>>>(A, lda, (int)M, (int)K, (int)M,
                                                                    (int)Kp, a, Kp);
        round_rows_kernel<cutlass::half_t, 1, kPatX1><<<gb, threads, 0, st>>>(
            B, ldb, (int)N, (int)K, (int)Np, (int)Kp, b, Kw);
        NMX_CUDA_TRY(cudaGetLastError());
        rc = tc::fp16t::run((int)M, (int)Np, (int)Kw, a, Kw, b, Kw, C, ldc, st, 0);
    } else {
        auto *a = reinterpret_cast<cutlass::bfloat16_t *>(a16);
        auto *b = reinterpret_cast<cutlass::bfloat16_t *>(b16);
        if (precision == NMX_PREC_BF16X3) {
            round_split_bf16_kernel<true><<<ga, threads, 0, st>>>(A, lda, (int)M, (int)K, (int)M,
                                                                  (int)Kp, a, Kw);
            round_rows_kernel<cutlass::bfloat16_t, 3, kPatX3B><<<gb, threads, 0, st>>>(
                B, ldb, (int)N, (int)K, (int)Np, (int)Kp, b, Kw);
        } else if (precision == NMX_PREC_BF16X6) {
            round_split6_bf16_kernel<true><<<ga, threads, 0, st>>>(A, lda, (int)M, (int)K, (int)M,
                                                                   (int)Kp, a, Kw);
            round_rows_kernel<cutlass::bfloat16_t, 6, kPatX6B><<<gb, threads, 0, st>>>(
                B, ldb, (int)N, (int)K, (int)Np, (int)Kp, b, Kw);
        } else {
            round_block_kernel<cutlass::bfloat16_t><<<ga, threads, 0, st>>>(A, lda, (int)M, (int)K,
                                                                            (int)M, (int)Kp, a, Kp);
            round_rows_kernel<cutlass::bfloat16_t, 1, kPatX1><<<gb, threads, 0, st>>>(
                B, ldb, (int)N, (int)K, (int)Np, (int)Kp, b, Kw);
        }
        NMX_CUDA_TRY(cudaGetLastError());
        rc = tc::bf16t::run((int)M, (int)Np, (int)Kw, a, Kw, b, Kw, C, ldc, st, 0);
    }
    if (rc) {
        set_error("tensor-core GEMM (B^T) %lldx%lldx%lld failed at step %d", (long long)M,
                  (long long)N, (long long)K, rc);
        return NMX_ERR_INTERNAL;
    }
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

size_t tc_gemm_workspace_bytes(int64_t M, int64_t N, int64_t K, int precision) {
    const int64_t Kp = up8(K) * split_factor(precision), Np = up8(N);
    return ((2 * (size_t)M * Kp + 255) & ~size_t(255)) + 2 * (size_t)Kp * Np + 512;
}

}  // namespace nmx

// ---- C ABI: the trailing-update primitive on its own ------------------------
extern "C" NMX_API int nmx_gemm_sub_f32(nmx_ctx ctx, int64_t M, int64_t N, int64_t K,
                                        const float *A, int64_t lda, const float *B, int64_t ldb,
                                        float *C, int64_t ldc, int precision, void *stream) {
    using namespace nmx;
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(M >= 0 && N >= 0 && K >= 0, 2, "negative size");
    NMX_ARG_CHECK(A != nullptr || M * K == 0, 5, "A is NULL");
    NMX_ARG_CHECK(lda >= std::max<int64_t>(1, K), 6, "lda < K");
    NMX_ARG_CHECK(B != nullptr || K * N == 0, 7, "B is NULL");
    NMX_ARG_CHECK(ldb >= std::max<int64_t>(1, N), 8, "ldb < N");
    NMX_ARG_CHECK(C != nullptr || M * N == 0, 9, "C is NULL");
    NMX_ARG_CHECK(ldc >= std::max<int64_t>(1, N), 10, "ldc < N");
    NMX_ARG_CHECK(precision == NMX_PREC_BF16 || precision == NMX_PREC_FP16 ||
                      precision == NMX_PREC_BF16X3 || precision == NMX_PREC_BF16X6,
                  11, "precision must be NMX_PREC_BF16, NMX_PREC_FP16, NMX_PREC_BF16X3 or "
                      "NMX_PREC_BF16X6");
    if (M == 0 || N == 0 || K == 0) return 0;
    DeviceGuard g(ctx->device);
    void *ws = nullptr;
    const size_t bytes = tc_gemm_workspace_bytes(M, N, K, precision);
    int rc = ctx->ensure_slot(kWsGemm16, bytes, &ws);
    if (rc) return rc;
    return tc_gemm_sub_f32(static_cast<cudaStream_t>(stream), precision, M, N, K, A, lda, B, ldb, C,
                           ldc, ws, bytes);
}
