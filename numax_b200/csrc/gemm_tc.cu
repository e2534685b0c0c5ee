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

#include "gemm_tc.cuh"

#pragma nv_diag_suppress 20012

namespace nmx {
namespace tc {

using namespace cute;

// One complete sm100 GEMM type per 16-bit input type, spelled at namespace
// scope (the host compiler rejects the dependent carve-out inside a class
// template).
#define NMX_TC_GEMM(NAME, ELEM)                                                                  \
    namespace NAME {                                                                             \
    using ElementA = ELEM;                                                                       \
    using ElementB = ELEM;                                                                       \
    using LayoutA = cutlass::layout::RowMajor; /* M x K, K contiguous */                         \
    using LayoutB = cutlass::layout::RowMajor; /* K x N, N contiguous (MN-major) */              \
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
                                                        void>;                                   \
    using Gemm = cutlass::gemm::device::GemmUniversalAdapter<Kernel>;                            \
    inline int run(int M, int N, int K, const void *A, int64_t lda, const void *B, int64_t ldb,  \
                   float *C, int64_t ldc, cudaStream_t st) {                                     \
        Kernel::StrideA sa{};                                                                    \
        Kernel::StrideB sb{};                                                                    \
        Kernel::StrideC sc{};                                                                    \
        Kernel::StrideD sd{};                                                                    \
        cute::get<0>(sa) = lda;                                                                  \
        cute::get<1>(sb) = ldb;                                                                  \
        cute::get<0>(sc) = ldc;                                                                  \
        cute::get<0>(sd) = ldc;                                                                  \
        Gemm::Arguments args{cutlass::gemm::GemmUniversalMode::kGemm,                            \
                             {M, N, K, 1},                                                       \
                             {static_cast<const ElementA *>(A), sa,                              \
                              static_cast<const ElementB *>(B), sb},                             \
                             {{-1.0f, 1.0f}, C, sc, C, sd}};                                     \
        Gemm g;                                                                                  \
        if (g.can_implement(args) != cutlass::Status::kSuccess) return 1;                        \
        if (Gemm::get_workspace_size(args) != 0) return 4;                                       \
        if (g.initialize(args, nullptr, st) != cutlass::Status::kSuccess) return 2;              \
        return g.run(st) == cutlass::Status::kSuccess ? 0 : 3;                                   \
    }                                                                                            \
    }

NMX_TC_GEMM(bf16, cutlass::bfloat16_t)
NMX_TC_GEMM(fp16, cutlass::half_t)
#undef NMX_TC_GEMM

}  // namespace tc

// fp32 block (rows x cols, ld) -> 16-bit dense block (ld_out), row-major.
template <typename Elem>
__global__ void round_block_kernel(const float *src, int64_t lds, int rows, int cols, Elem *dst,
                                   int64_t ldd) {
    const int64_t e = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (int64_t)rows * cols) return;
    const int r = (int)(e / cols), c = (int)(e - (int64_t)r * cols);
    dst[(int64_t)r * ldd + c] = Elem(src[(int64_t)r * lds + c]);
}

int tc_gemm_sub_f32(cudaStream_t st, int precision, int64_t M, int64_t N, int64_t K, const float *A,
                    int64_t lda, const float *B, int64_t ldb, float *C, int64_t ldc, void *ws,
                    size_t ws_bytes) {
    if (M <= 0 || N <= 0 || K <= 0) return 0;
    const int64_t ldk = (K + 7) / 8 * 8, ldn = (N + 7) / 8 * 8;
    const size_t need = 2 * (size_t)(M * ldk + K * ldn) + 256;
    if (need > ws_bytes) {
        set_error("tensor-core update needs %zu B of workspace, have %zu", need, ws_bytes);
        return NMX_ERR_INTERNAL;
    }
    if ((ldc % 4) != 0 || (reinterpret_cast<uintptr_t>(C) % 16) != 0) {
        set_error("tensor-core update: C must be 16-byte aligned with ldc % 4 == 0");
        return NMX_ERR_INTERNAL;
    }
    auto *a16 = static_cast<unsigned char *>(ws);
    auto *b16 = a16 + ((2 * (size_t)M * ldk + 255) & ~size_t(255));
    const int threads = 256;
    int rc;
    if (precision == NMX_PREC_FP16) {
        round_block_kernel<cutlass::half_t><<<(unsigned)ceil_div(M * K, threads), threads, 0, st>>>(
            A, lda, (int)M, (int)K, reinterpret_cast<cutlass::half_t *>(a16), ldk);
        round_block_kernel<cutlass::half_t><<<(unsigned)ceil_div(K * N, threads), threads, 0, st>>>(
            B, ldb, (int)K, (int)N, reinterpret_cast<cutlass::half_t *>(b16), ldn);
        NMX_CUDA_TRY(cudaGetLastError());
        rc = tc::fp16::run((int)M, (int)N, (int)K, a16, ldk, b16, ldn, C, ldc, st);
    } else {
        round_block_kernel<cutlass::bfloat16_t>
            <<<(unsigned)ceil_div(M * K, threads), threads, 0, st>>>(
                A, lda, (int)M, (int)K, reinterpret_cast<cutlass::bfloat16_t *>(a16), ldk);
        round_block_kernel<cutlass::bfloat16_t>
            <<<(unsigned)ceil_div(K * N, threads), threads, 0, st>>>(
                B, ldb, (int)K, (int)N, reinterpret_cast<cutlass::bfloat16_t *>(b16), ldn);
        NMX_CUDA_TRY(cudaGetLastError());
        rc = tc::bf16::run((int)M, (int)N, (int)K, a16, ldk, b16, ldn, C, ldc,
                                                   st);
    }
    if (rc) {
        set_error("tensor-core GEMM %lldx%lldx%lld failed at step %d", (long long)M, (long long)N,
                  (long long)K, rc);
        return NMX_ERR_INTERNAL;
    }
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

size_t tc_gemm_workspace_bytes(int64_t M, int64_t N, int64_t K) {
    const int64_t ldk = (K + 7) / 8 * 8, ldn = (N + 7) / 8 * 8;
    return 2 * (size_t)(M * ldk + K * ldn) + 512;
}

}  // namespace nmx
