// Tensor-core (tcgen05, BF16/FP16 in, FP32 accumulate) trailing update used
// by the mixed-precision factorizations.  Implemented in gemm_tc.cu.
#pragma once

#include "nmx_common.cuh"

#ifndef NMX_PREC_BF16
#define NMX_PREC_BF16 1
#define NMX_PREC_FP16 2
#define NMX_PREC_BF16X3 3
#define NMX_PREC_BF16X6 4
#endif

namespace nmx {

// C[M x N] -= round(A)[M x K] * round(B)[K x N], fp32 row-major operands,
// rounded to BF16 (precision = NMX_PREC_BF16) or FP16, or split into 2 / 3
// BF16 pieces (NMX_PREC_BF16X3 / NMX_PREC_BF16X6), into `ws` first.
// C must be 16-byte aligned with ldc % 4 == 0.  sm_limit > 0 keeps the GEMM
// on at most that many SMs.
// b_kmajor: B is stored N x K (ldb), i.e. C -= A B^T.
int tc_gemm_sub_f32(cudaStream_t st, int precision, int64_t M, int64_t N, int64_t K, const float *A,
                    int64_t lda, const float *B, int64_t ldb, float *C, int64_t ldc, void *ws,
                    size_t ws_bytes, int sm_limit = 0, bool b_kmajor = false);
int tc_gemm_sub_bt_f32(cudaStream_t st, int precision, int64_t M, int64_t N, int64_t K,
                       const float *A, int64_t lda, const float *B, int64_t ldb, float *C,
                       int64_t ldc, void *ws, size_t ws_bytes);

// Workspace tc_gemm_sub_f32 needs for an M x N x K update.
size_t tc_gemm_workspace_bytes(int64_t M, int64_t N, int64_t K, int precision = NMX_PREC_BF16);

}  // namespace nmx
