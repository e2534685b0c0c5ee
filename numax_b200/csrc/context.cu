// Context lifecycle and error reporting for libnmxla.so.
#include <cstring>

#include "nmx_common.cuh"

namespace nmx {

static thread_local char g_last_error[1024] = {0};

void set_error(const char *fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_last_error, sizeof(g_last_error), fmt, ap);
    va_end(ap);
}

void clear_error() { g_last_error[0] = 0; }

int ctx_lookahead_streams(nmx_ctx ctx) {
    if (ctx->la_stream[0]) return 0;
    int least = 0, greatest = 0;
    NMX_CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    // All four objects or none: the context keeps them only when every one
    // was created.
    cudaStream_t s[2] = {};
    cudaEvent_t e[2] = {};
    cudaError_t err = cudaStreamCreateWithPriority(&s[0], cudaStreamNonBlocking, greatest);
    if (err == cudaSuccess) err = cudaStreamCreateWithPriority(&s[1], cudaStreamNonBlocking, least);
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e[0], cudaEventDisableTiming);
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e[1], cudaEventDisableTiming);
    if (err != cudaSuccess) {
        for (int i = 0; i < 2; ++i) {
            if (s[i]) cudaStreamDestroy(s[i]);
            if (e[i]) cudaEventDestroy(e[i]);
        }
        set_error("look-ahead streams: %s", cudaGetErrorString(err));
        return NMX_ERR_CUDA;
    }
    for (int i = 0; i < 2; ++i) {
        ctx->la_stream[i] = s[i];
        ctx->la_event[i] = e[i];
    }
    return 0;
}

}  // namespace nmx

int nmx_context::ensure_workspace(size_t bytes) {
    if (bytes <= workspace_bytes) return 0;
    if (workspace) cudaFree(workspace);
    workspace = nullptr;
    workspace_bytes = 0;
    size_t rounded = (bytes + (1 << 20) - 1) & ~size_t((1 << 20) - 1);
    cudaError_t e = cudaMalloc(&workspace, rounded);
    if (e != cudaSuccess) {
        nmx::set_error("workspace cudaMalloc(%zu): %s", rounded, cudaGetErrorString(e));
        return NMX_ERR_ALLOC;
    }
    workspace_bytes = rounded;
    return 0;
}

int nmx_context::ensure_slot(int slot, size_t bytes, void **out) {
    if (slot < 0 || slot >= kSlots) {
        nmx::set_error("bad workspace slot %d", slot);
        return NMX_ERR_INTERNAL;
    }
    if (bytes > slot_bytes[slot]) {
        if (slot_ptr[slot]) cudaFree(slot_ptr[slot]);
        slot_ptr[slot] = nullptr;
        slot_bytes[slot] = 0;
        size_t rounded = (bytes + (1 << 20) - 1) & ~size_t((1 << 20) - 1);
        cudaError_t e = cudaMalloc(&slot_ptr[slot], rounded);
        if (e != cudaSuccess) {
            nmx::set_error("workspace slot %d cudaMalloc(%zu): %s", slot, rounded,
                           cudaGetErrorString(e));
            return NMX_ERR_ALLOC;
        }
        slot_bytes[slot] = rounded;
    }
    *out = slot_ptr[slot];
    return 0;
}

extern "C" {

const char *nmx_last_error_string(void) { return nmx::g_last_error; }

int nmx_version(void) { return 100; }

int nmx_create(int device, nmx_ctx *out) {
    NMX_ARG_CHECK(out != nullptr, 2, "out is NULL");
    *out = nullptr;
    int ndev = 0;
    NMX_CUDA_TRY(cudaGetDeviceCount(&ndev));
    NMX_ARG_CHECK(device >= 0 && device < ndev, 1, "no such CUDA device");
    nmx::DeviceGuard g(device);
    cudaDeviceProp prop;
    NMX_CUDA_TRY(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) {
        nmx::set_error("device %d is sm_%d%d; libnmxla is built for sm_100a only", device,
                       prop.major, prop.minor);
        return NMX_ERR_UNSUPPORTED;
    }
    nmx_context *ctx = new (std::nothrow) nmx_context();
    if (!ctx) return NMX_ERR_ALLOC;
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    ctx->cc_major = prop.major;
    ctx->cc_minor = prop.minor;
    ctx->smem_optin = prop.sharedMemPerBlockOptin;
    *out = ctx;
    nmx::clear_error();
    return 0;
}

// Tuning knobs.  Keys: "lu.leaf_ctas", "ir.trsv_ctas" (0 = automatic).
static int64_t *tune_slot(nmx_ctx ctx, const char *key) {
    if (!key) return nullptr;
    if (!std::strcmp(key, "lu.leaf_ctas")) return &ctx->tune_lu_leaf_ctas;
    if (!std::strcmp(key, "ir.trsv_ctas")) return &ctx->tune_ir_trsv_ctas;
    if (!std::strcmp(key, "lu.cluster")) return &ctx->tune_lu_cluster;
    if (!std::strcmp(key, "ir.tc_min")) return &ctx->tune_ir_tc_min;
    if (!std::strcmp(key, "lu.leaf_w")) return &ctx->tune_lu_leaf_w;
    if (!std::strcmp(key, "lu.tournament")) return &ctx->tune_lu_tournament;
    if (!std::strcmp(key, "lu.lookahead")) return &ctx->tune_lu_lookahead;
    if (!std::strcmp(key, "lu.panel_sms")) return &ctx->tune_lu_panel_sms;
    return nullptr;
}

int nmx_tune_set(nmx_ctx ctx, const char *key, int64_t value) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    int64_t *slot = tune_slot(ctx, key);
    NMX_ARG_CHECK(slot != nullptr, 2, "unknown tuning key");
    NMX_ARG_CHECK(value >= -1, 3, "value must be >= -1");
    *slot = value;
    return 0;
}

int nmx_tune_get(nmx_ctx ctx, const char *key, int64_t *value) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    int64_t *slot = tune_slot(ctx, key);
    NMX_ARG_CHECK(slot != nullptr, 2, "unknown tuning key");
    NMX_ARG_CHECK(value != nullptr, 3, "value is NULL");
    *value = *slot;
    return 0;
}

int nmx_synchronize(nmx_ctx ctx, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    nmx::DeviceGuard g(ctx->device);
    NMX_CUDA_TRY(cudaStreamSynchronize(static_cast<cudaStream_t>(stream)));
    return 0;
}

int nmx_memcpy_to_host(nmx_ctx ctx, void *dst, const void *src, int64_t bytes, void *stream) {
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(dst != nullptr || bytes == 0, 2, "dst is NULL");
    NMX_ARG_CHECK(src != nullptr || bytes == 0, 3, "src is NULL");
    NMX_ARG_CHECK(bytes >= 0, 4, "bytes < 0");
    if (bytes == 0) return 0;
    nmx::DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    NMX_CUDA_TRY(cudaMemcpyAsync(dst, src, (size_t)bytes, cudaMemcpyDeviceToHost, st));
    NMX_CUDA_TRY(cudaStreamSynchronize(st));
    return 0;
}

int nmx_destroy(nmx_ctx ctx) {
    if (!ctx) return 0;
    {
        nmx::DeviceGuard g(ctx->device);
        if (ctx->workspace) cudaFree(ctx->workspace);
        for (int i = 0; i < nmx_context::kSlots; ++i)
            if (ctx->slot_ptr[i]) cudaFree(ctx->slot_ptr[i]);
        for (int i = 0; i < 2; ++i) {
            if (ctx->la_stream[i]) cudaStreamDestroy(ctx->la_stream[i]);
            if (ctx->la_event[i]) cudaEventDestroy(ctx->la_event[i]);
        }
        for (void *p : ctx->npy_pinned) cudaFreeHost(p);
        for (cudaEvent_t e : ctx->npy_event) cudaEventDestroy(e);
    }
    delete ctx;
    return 0;
}

}  // extern "C"
