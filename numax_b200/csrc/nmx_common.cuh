// Shared internals of libnmxla.so: error reporting, the context, small
// device helpers.  Not part of the public ABI (include/nmx_la.h is).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cstdarg>
#include <cstdio>
#include <string>
#include <vector>

#include "../../include/nmx_la.h"

namespace nmx {

// ---- error reporting --------------------------------------------------------

void set_error(const char *fmt, ...);
void clear_error();

#define NMX_CUDA_TRY(expr)                                                              \
    do {                                                                                \
        cudaError_t _e = (expr);                                                        \
        if (_e != cudaSuccess) {                                                        \
            ::nmx::set_error("%s:%d: %s -> %s", __FILE__, __LINE__, #expr,               \
                             cudaGetErrorString(_e));                                   \
            return NMX_ERR_CUDA;                                                        \
        }                                                                               \
    } while (0)

#define NMX_ARG_CHECK(cond, idx, msg)                                                   \
    do {                                                                                \
        if (!(cond)) {                                                                  \
            ::nmx::set_error("argument %d: %s", (idx), (msg));                          \
            return -(idx);                                                              \
        }                                                                               \
    } while (0)

// Propagate a nonzero status.
#define NMX_TRY(expr)           \
    do {                        \
        const int _rc = (expr); \
        if (_rc) return _rc;    \
    } while (0)

// Restores the caller's current device on scope exit.
struct DeviceGuard {
    int prev = -1;
    bool ok = true;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) ok = cudaSetDevice(dev) == cudaSuccess;
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

}  // namespace nmx

// The context: device, SM count, a grow-only workspace owned for the
// context's lifetime (numax allocates per call, numax/linalg/lu.mojo:582-584;
// here the context keeps it so repeated calls allocate nothing).
struct nmx_context {
    int device = 0;
    int sm_count = 0;
    int cc_major = 0, cc_minor = 0;
    size_t smem_optin = 0;
    void *workspace = nullptr;
    size_t workspace_bytes = 0;
    // The look-ahead LU's panel (high priority) and update streams and the
    // events that order them, created on first use.
    cudaStream_t la_stream[2] = {};
    cudaEvent_t la_event[2] = {};
    // Tuning knobs (nmx_tune_set / nmx_tune_get); 0 means "automatic".
    int64_t tune_lu_leaf_ctas = 0;    // CTAs of the cooperative LU leaf panel
    int64_t tune_ir_trsv_ctas = 0;    // CTAs of the persistent triangular solves
    int64_t tune_lu_cluster = -1;     // cap on the LU cluster leaf's CTAs (-1: none, 0: off)
    int64_t tune_lu_leaf_w = 0;       // widest LU leaf panel (0: 32; multiple of 8, <= 64)
    int64_t tune_ir_tc_min = -1;      // smallest GEMM inner dimension on the tensor cores (-1: 256)
    int64_t tune_lu_tournament = -1;  // tournament-pivoting FP32 leaves (-1: IR only, 0: never, 1: also nmx_getrf_f32)
    int64_t tune_lu_lookahead = -1;   // look-ahead panel width of the LU (-1: 256, 0: off)
    int64_t tune_lu_panel_sms = -1;   // SMs the look-ahead keeps free of the update GEMMs (-1, 0: none)
    // Grow-only named device buffers, one per use, kept for the context's life.
    static constexpr int kSlots = 12;
    void *slot_ptr[kSlots] = {};
    size_t slot_bytes[kSlots] = {};
    // Pinned host staging of the .npy load/save pipeline and, per buffer, the
    // event of the copy that last used it (grown on first use).
    std::vector<void *> npy_pinned;
    std::vector<cudaEvent_t> npy_event;
    // Returns a device buffer of at least `bytes`, reusing the context's.
    int ensure_workspace(size_t bytes);
    // Same for slot `slot` (see nmx::WsSlot); *out receives the buffer.
    int ensure_slot(int slot, size_t bytes, void **out);
};

namespace nmx {
enum WsSlot {
    kWsLeaf = 0,
    kWsGemm16 = 1,
    kWsWork = 2,
    kWsVec = 3,
    kWsKrylov = 4,
    kWsInv = 5,
    kWsCalu = 6,
    kWsGemm16Panel = 7,
    kWsWork64 = 8,  // FP64 factors of the refinement's last precision level
    kWsBest = 9,    // the refinement's best iterate
    kWsAux = 10,    // inverse's factor copy, PLU's permutation
    kWsEig = 11     // the symmetric eigensolver's work copy and divide-and-conquer buffers
};
}

namespace nmx {

// ---- device helpers ---------------------------------------------------------

// guard_nonzero(x, floor) = copysign(max_of(|x|, floor), x), with numax's
// max_of being an exact selection where |x| >= floor wins
// (numax/core/numeric.mojo:263-366).  A NaN propagates.
template <typename T>
__device__ __forceinline__ T guard_nonzero(T x, T floor_) {
    T ax = fabs(x);
    T m = (ax >= floor_ || ax != ax) ? ax : floor_;
    return copysign(m, x);
}

template <typename T>
struct pivot_floor;
template <>
struct pivot_floor<double> {
    static constexpr double value = 1e-30;
};
template <>
struct pivot_floor<float> {
    static constexpr float value = 1e-30f;
};

__host__ __device__ __forceinline__ int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

}  // namespace nmx
