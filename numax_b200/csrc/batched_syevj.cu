// Batched uneven-size symmetric eigensolver, parallel-order Jacobi (sm_100a).
//
// Replaces numax's Array-tier `eigh` run one matrix per GPU thread
// (numax/linalg/_array/eigen.mojo:316-392, launched through `map` in
// examples/advanced/quantum_well.mojo:149-157): cyclic-by-row Jacobi with a
// fixed 12 sweeps out of spilling registers.  Here each matrix (n <= 64,
// float32 data) is staged into shared memory and worked by a group of
// threads -- one warp for n <= 32, a 128-thread CTA above -- with the
// round-robin ordering: each sweep is m-1 rounds (m = n rounded up to even)
// of m/2 disjoint rotations applied at once.  With disjoint pairs the
// similarity J^T A J splits into independent 2x2 blocks B' = R_k^T B R_l, so
// a round is one pass over the blocks plus one over the rows of V.
//
// Rotation angles are computed in float64 with numax's formula
// (numax/linalg/_array/eigen.mojo:34-75): t = sign(d) 2 a_pq /
// (|d| + sqrt(d^2 + 4 a_pq^2)), d = a_qq - a_pp, c = 1/sqrt(1+t^2), s = t c.
// The sweep loop stops when the float64 off-diagonal norm falls to
// tol * ||A||_F (or after max_sweeps), instead of numax's fixed 12.
#include <algorithm>
#include <numeric>
#include <vector>

#include "nmx_common.cuh"

namespace nmx {

constexpr int kSyevjMaxN = 64;

struct BatchedSyevjArgs {
    const int32_t *order;
    const int32_t *ns;
    const int64_t *a_off;
    const int64_t *w_off;
    const float *A;
    float *W;
    float *V;
    int32_t *sweeps;
    double tol;
    int max_sweeps;
    int sort;
};

// Index at tournament position `pos` in round `r` (m players, player 0 fixed).
__device__ __forceinline__ int tourney(int pos, int r, int m) {
    return pos == 0 ? 0 : (pos - 1 + r) % (m - 1) + 1;
}

// Group-level barrier: a warp for G == 32, else the whole CTA (G == NT).
template <int G>
__device__ __forceinline__ void group_sync() {
    if (G == 32)
        __syncwarp();
    else
        __syncthreads();
}

// A matrix of order n is worked on at the even order m = n + (n & 1): an odd
// n gets a zero row and column (and a zero row/column in V), whose pairs
// always rotate by the identity (a_pq = 0 gives t = 0), so every pair of a
// round is a full 2x2 update without branches.  Row pitch m_max + 1 (odd).
__host__ __device__ inline int syevj_even(int n) { return n + (n & 1); }
__host__ __device__ inline int syevj_ld(int nmax) { return syevj_even(nmax) + 1; }

// Per-group shared-memory floats for matrices up to nmax: A and V (m_max
// rows of pitch ld), the round's rotations (float2 c, s) and pairs (int4
// p, q, p*ld, q*ld), and a float64 reduction scratch.
__host__ __device__ inline int syevj_group_floats(int nmax) {
    const int m = syevj_even(nmax), half = m / 2 + 1;
    return 2 * m * syevj_ld(nmax) + half * 2 + half * 4 + 2 * 64 + 4;
}

template <int G>
__device__ void syevj_one(const BatchedSyevjArgs &args, int mi, float *As, float *Vs, float2 *csf,
                          int4 *pqo, double *red, int gt, int ld) {
    const int n = args.ns[mi];
    const int m = syevj_even(n);
    const int half = m / 2;
    const float *A = args.A + args.a_off[mi];
    float *V = args.V + args.a_off[mi];
    float *W = args.W + args.w_off[mi];

    for (int e = gt; e < m * m; e += G) {
        const int i = e / m, j = e - i * m;
        As[i * ld + j] = (i < n && j < n) ? A[i * n + j] : 0.f;
        Vs[i * ld + j] = (i == j && i < n) ? 1.f : 0.f;
    }
    group_sync<G>();

    int sweep = 0;
    for (;; ++sweep) {
        // float64 off-diagonal and total Frobenius norms.
        double off = 0.0, tot = 0.0;
        for (int e = gt; e < n * n; e += G) {
            int i = e / n, j = e - i * n;
            double v = As[i * ld + j];
            tot += v * v;
            if (i != j) off += v * v;
        }
        for (int o = 16; o > 0; o >>= 1) {
            off += __shfl_xor_sync(0xffffffffu, off, o);
            tot += __shfl_xor_sync(0xffffffffu, tot, o);
        }
        if (G > 32) {
            if ((gt & 31) == 0) {
                red[2 * (gt >> 5)] = off;
                red[2 * (gt >> 5) + 1] = tot;
            }
            group_sync<G>();
            off = tot = 0.0;
            for (int w = 0; w < G / 32; ++w) {
                off += red[2 * w];
                tot += red[2 * w + 1];
            }
            group_sync<G>();
        }
        if (!(off > args.tol * args.tol * tot) || sweep >= args.max_sweeps) break;

        for (int r = 0; r < m - 1; ++r) {
            // Pairs and float64 rotations for this round (the padding pair of
            // an odd n gets c = 1, s = 0).
            for (int k = gt; k < half; k += G) {
                const int a = tourney(k, r, m), b = tourney(m - 1 - k, r, m);
                const int p = min(a, b), q = max(a, b);
                // numax's angle, evaluated with reciprocal square roots and
                // one correctly rounded reciprocal (the chain of two square
                // roots and two divisions is the round's latency).
                const double apq = As[p * ld + q], app = As[p * ld + p], aqq = As[q * ld + q];
                const double d = aqq - app;
                const double two = 2.0 * apq;
                const double r2 = d * d + two * two;
                const double radius = r2 > 0.0 ? r2 * rsqrt(r2) : 0.0;
                const double safe = guard_nonzero(fabs(d) + radius, 1e-30);
                const double t = copysign(1.0, d) * two * __drcp_rn(safe);
                const double c = rsqrt(1.0 + t * t);
                csf[k] = make_float2((float)c, (float)(t * c));
                pqo[k] = make_int4(p, q, p * ld, q * ld);
            }
            group_sync<G>();
            // 2x2 blocks B' = R_k^T B R_l: lane = column pair l, warps = row
            // pairs k.  The rotations were formed in float64; they are applied
            // to the float32 data in float32.
            {
                constexpr int NWG = G / 32;
                const int lane = gt & 31, wg = gt >> 5;
                if (lane < half) {
                    const int4 cu = pqo[lane];
                    const float2 cc = csf[lane];
#pragma unroll 4
                    for (int kr = wg; kr < half; kr += NWG) {
                        const int4 ru = pqo[kr];
                        const float2 rc = csf[kr];
                        const float b00 = As[ru.z + cu.x], b01 = As[ru.z + cu.y];
                        const float b10 = As[ru.w + cu.x], b11 = As[ru.w + cu.y];
                        // rows: [c -s; s c] from the left, columns: [c s; -s c] from the right
                        const float r00 = rc.x * b00 - rc.y * b10, r01 = rc.x * b01 - rc.y * b11;
                        const float r10 = rc.y * b00 + rc.x * b10, r11 = rc.y * b01 + rc.x * b11;
                        const bool own = kr == lane;  // the annihilated pair
                        As[ru.z + cu.x] = cc.x * r00 - cc.y * r01;
                        As[ru.z + cu.y] = own ? 0.f : cc.y * r00 + cc.x * r01;
                        As[ru.w + cu.x] = own ? 0.f : cc.x * r10 - cc.y * r11;
                        As[ru.w + cu.y] = cc.y * r10 + cc.x * r11;
                    }
                    // V := V J: warps = rows of V, lane = column pair.
#pragma unroll 4
                    for (int i = wg; i < n; i += NWG) {
                        const float vp = Vs[i * ld + cu.x], vq = Vs[i * ld + cu.y];
                        Vs[i * ld + cu.x] = cc.x * vp - cc.y * vq;
                        Vs[i * ld + cu.y] = cc.y * vp + cc.x * vq;
                    }
                }
            }
            group_sync<G>();
        }
    }

    // Eigenvalues: the diagonal, optionally sorted ascending with V's columns.
    if (args.sort) {
        for (int i = gt; i < n; i += G) {
            float wi = As[i * ld + i];
            int rank = 0;
            for (int j = 0; j < n; ++j) {
                float wj = As[j * ld + j];
                rank += (wj < wi) || (wj == wi && j < i);
            }
            W[rank] = wi;
            for (int r = 0; r < n; ++r) V[(int64_t)r * n + rank] = Vs[r * ld + i];
        }
    } else {
        for (int i = gt; i < n; i += G) W[i] = As[i * ld + i];
        for (int e = gt; e < n * n; e += G) {
            int i = e / n, j = e - i * n;
            V[e] = Vs[i * ld + j];
        }
    }
    if (gt == 0 && args.sweeps) args.sweeps[mi] = sweep;
    group_sync<G>();
}

template <int NT, int G>
__global__ void __launch_bounds__(NT) syevj_batched_kernel(BatchedSyevjArgs args, int begin, int end,
                                                           int nmax, int *counter) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    constexpr int NG = NT / G;
    const int g = threadIdx.x / G, gt = threadIdx.x - g * G;
    const int ld = syevj_ld(nmax), mmax = syevj_even(nmax), hmax = mmax / 2 + 1;
    const int per_group = syevj_group_floats(nmax);
    float *base = reinterpret_cast<float *>(smem_raw) + (size_t)g * ((per_group + 3) & ~3);
    float *As = base;
    float *Vs = As + mmax * ld;
    // 16-byte aligned tables after A and V.
    int4 *pqo = reinterpret_cast<int4 *>((reinterpret_cast<uintptr_t>(Vs + mmax * ld) + 15) & ~uintptr_t(15));
    float2 *csf = reinterpret_cast<float2 *>(pqo + hmax);
    double *red = reinterpret_cast<double *>(csf + hmax);
    __shared__ int s_item[NG];
    for (;;) {
        if (gt == 0) s_item[g] = atomicAdd(counter, 1);
        group_sync<G>();
        const int item = begin + s_item[g];
        group_sync<G>();
        if (item >= end) break;
        syevj_one<G>(args, args.order[item], As, Vs, csf, pqo, red, gt, ld);
    }
}

}  // namespace nmx

struct nmx_syevj_plan_s {
    int device = 0;
    int64_t count = 0;
    int64_t a_elems = 0, w_elems = 0;
    void *dev = nullptr;
    int32_t *d_order = nullptr, *d_n = nullptr, *d_counters = nullptr;
    int64_t *d_aoff = nullptr, *d_woff = nullptr;
    struct Bucket {
        int begin, end, nmax, threads, group, grid;
        size_t smem;
    };
    std::vector<Bucket> buckets;
    // CUDA graph of one run, for the arguments in graph_key.
    cudaGraphExec_t graph = nullptr;
    const void *graph_key[4] = {nullptr, nullptr, nullptr, nullptr};
    double graph_tol = -1.0;
    int graph_max_sweeps = -1, graph_sort = -1;
};

namespace nmx {

template <int NT, int G>
static int syevj_configure(nmx_ctx ctx, nmx_syevj_plan_s::Bucket &b) {
    auto kern = syevj_batched_kernel<NT, G>;
    b.threads = NT;
    b.group = G;
    size_t per_group = ((size_t)syevj_group_floats(b.nmax) + 3) & ~size_t(3);
    b.smem = sizeof(float) * per_group * (NT / G) + 64;
    cudaFuncAttributes fa;
    NMX_CUDA_TRY(cudaFuncGetAttributes(&fa, kern));
    if (b.smem + fa.sharedSizeBytes > ctx->smem_optin) {
        set_error("syevj bucket nmax=%d needs %zu B shared memory", b.nmax, b.smem);
        return NMX_ERR_UNSUPPORTED;
    }
    NMX_CUDA_TRY(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)(ctx->smem_optin - fa.sharedSizeBytes)));
    int per_sm = 0;
    NMX_CUDA_TRY(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, b.smem));
    if (per_sm < 1) {
        set_error("syevj bucket nmax=%d does not fit an SM", b.nmax);
        return NMX_ERR_UNSUPPORTED;
    }
    int64_t groups = (int64_t)per_sm * ctx->sm_count * (NT / G);
    int64_t work = b.end - b.begin;
    b.grid = (int)std::max<int64_t>(1, std::min<int64_t>(ceil_div(work, NT / G), groups / (NT / G)));
    return 0;
}

// The (threads, group) shapes a bucket can run with: a warp per matrix
// (group 32) in CTAs of 1..8 warps, or a whole CTA per matrix.
static const int kSyevjShapes[][2] = {{128, 32}, {64, 32}, {256, 32}, {32, 32},
                                      {64, 64}, {128, 128}, {256, 256}};

static int syevj_configure_shape(nmx_ctx ctx, nmx_syevj_plan_s::Bucket &b, int threads, int group) {
    switch (threads * 1000 + group) {
#define NMX_SHAPE(NT, G) \
    case NT * 1000 + G:  \
        return syevj_configure<NT, G>(ctx, b);
        NMX_SHAPE(128, 32)
        NMX_SHAPE(64, 32)
        NMX_SHAPE(256, 32)
        NMX_SHAPE(32, 32)
        NMX_SHAPE(64, 64)
        NMX_SHAPE(128, 128)
        NMX_SHAPE(256, 256)
#undef NMX_SHAPE
        default:
            set_error("unsupported eigh shape %d threads / group %d", threads, group);
            return NMX_ERR_INTERNAL;
    }
}

static int syevj_launch(const BatchedSyevjArgs &args, const nmx_syevj_plan_s::Bucket &b,
                        int *counter, cudaStream_t st) {
    switch (b.threads * 1000 + b.group) {
#define NMX_SHAPE(NT, G)                                                                          \
    case NT * 1000 + G:                                                                           \
        syevj_batched_kernel<NT, G><<<b.grid, NT, b.smem, st>>>(args, b.begin, b.end, b.nmax, counter); \
        break;
        NMX_SHAPE(128, 32)
        NMX_SHAPE(64, 32)
        NMX_SHAPE(256, 32)
        NMX_SHAPE(32, 32)
        NMX_SHAPE(64, 64)
        NMX_SHAPE(128, 128)
        NMX_SHAPE(256, 256)
#undef NMX_SHAPE
        default:
            set_error("unsupported eigh shape %d threads / group %d", b.threads, b.group);
            return NMX_ERR_INTERNAL;
    }
    NMX_CUDA_TRY(cudaGetLastError());
    return 0;
}

static int syevj_run(nmx_syevj_plan_s *plan, const BatchedSyevjArgs &args, cudaStream_t st) {
    NMX_CUDA_TRY(cudaMemsetAsync(plan->d_counters, 0, sizeof(int32_t) * plan->buckets.size(), st));
    for (size_t bi = 0; bi < plan->buckets.size(); ++bi)
        NMX_TRY(syevj_launch(args, plan->buckets[bi], plan->d_counters + bi, st));
    return 0;
}

}  // namespace nmx

extern "C" {

NMX_API int nmx_syevj_batched_plan(nmx_ctx ctx, int64_t count, const int32_t *n_host,
                                   nmx_syevj_plan *out) {
    using namespace nmx;
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(count >= 0 && count < (int64_t(1) << 31), 2, "count out of range");
    NMX_ARG_CHECK(n_host != nullptr || count == 0, 3, "n_host is NULL");
    NMX_ARG_CHECK(out != nullptr, 4, "out is NULL");
    for (int64_t i = 0; i < count; ++i)
        NMX_ARG_CHECK(n_host[i] >= 1 && n_host[i] <= kSyevjMaxN, 3, "every n_i must be in 1..64");
    *out = nullptr;
    DeviceGuard g(ctx->device);
    auto *p = new (std::nothrow) nmx_syevj_plan_s();
    if (!p) return NMX_ERR_ALLOC;
    p->device = ctx->device;
    p->count = count;
    std::vector<int64_t> aoff(count), woff(count);
    int64_t a = 0, w = 0;
    for (int64_t i = 0; i < count; ++i) {
        aoff[i] = a;
        woff[i] = w;
        a += (int64_t)n_host[i] * n_host[i];
        w += n_host[i];
    }
    p->a_elems = a;
    p->w_elems = w;
    std::vector<int32_t> order(count);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int32_t x, int32_t y) { return n_host[x] > n_host[y]; });
    int64_t pos = 0;
    // Bucket 0: n in 33..64, one 128-thread CTA per matrix; bucket 1: n <= 32,
    // one warp per matrix, four per CTA.
    int64_t begin = pos;
    while (pos < count && n_host[order[pos]] > 32) ++pos;
    if (pos > begin) p->buckets.push_back({(int)begin, (int)pos, n_host[order[begin]], 128, 128, 0, 0});
    begin = pos;
    pos = count;
    if (pos > begin) p->buckets.push_back({(int)begin, (int)pos, n_host[order[begin]], 128, 32, 0, 0});
    size_t nb = p->buckets.size();
    size_t bytes = sizeof(int64_t) * 2 * count + sizeof(int32_t) * (2 * count + nb + 1) + 64;
    cudaError_t e = cudaMalloc(&p->dev, bytes);
    if (e != cudaSuccess) {
        delete p;
        set_error("plan cudaMalloc: %s", cudaGetErrorString(e));
        return NMX_ERR_ALLOC;
    }
    p->d_aoff = static_cast<int64_t *>(p->dev);
    p->d_woff = p->d_aoff + count;
    p->d_order = reinterpret_cast<int32_t *>(p->d_woff + count);
    p->d_n = p->d_order + count;
    p->d_counters = p->d_n + count;
    int rc = 0;
    if (count &&
        (cudaMemcpy(p->d_aoff, aoff.data(), 8 * count, cudaMemcpyHostToDevice) ||
         cudaMemcpy(p->d_woff, woff.data(), 8 * count, cudaMemcpyHostToDevice) ||
         cudaMemcpy(p->d_order, order.data(), 4 * count, cudaMemcpyHostToDevice) ||
         cudaMemcpy(p->d_n, n_host, 4 * count, cudaMemcpyHostToDevice))) {
        set_error("syevj plan upload failed");
        rc = NMX_ERR_CUDA;
    }
    for (auto &b : p->buckets) {
        if (rc) break;
        rc = b.group == 32 ? syevj_configure<128, 32>(ctx, b) : syevj_configure<128, 128>(ctx, b);
    }
    if (rc) {
        cudaFree(p->dev);
        delete p;
        return rc;
    }
    *out = p;
    return 0;
}

NMX_API int nmx_syevj_plan_destroy(nmx_syevj_plan plan) {
    if (!plan) return 0;
    nmx::DeviceGuard g(plan->device);
    if (plan->graph) cudaGraphExecDestroy(plan->graph);
    if (plan->dev) cudaFree(plan->dev);
    delete plan;
    return 0;
}

NMX_API int nmx_syevj_plan_sizes(nmx_syevj_plan plan, int64_t *a_elems, int64_t *w_elems) {
    NMX_ARG_CHECK(plan != nullptr, 1, "plan is NULL");
    if (a_elems) *a_elems = plan->a_elems;
    if (w_elems) *w_elems = plan->w_elems;
    return 0;
}

NMX_API int nmx_syevj_batched_f32(nmx_ctx ctx, nmx_syevj_plan plan, const float *A, float *W,
                                  float *V, int32_t *sweeps, double tol, int max_sweeps, int sort,
                                  void *stream) {
    using namespace nmx;
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(plan != nullptr, 2, "plan is NULL");
    NMX_ARG_CHECK(A != nullptr || plan->count == 0, 3, "A is NULL");
    NMX_ARG_CHECK(W != nullptr || plan->count == 0, 4, "W is NULL");
    NMX_ARG_CHECK(V != nullptr || plan->count == 0, 5, "V is NULL");
    NMX_ARG_CHECK(tol >= 0.0, 7, "tol must be >= 0");
    NMX_ARG_CHECK(max_sweeps >= 0 && max_sweeps <= 1000, 8, "max_sweeps must be in 0..1000");
    if (plan->count == 0) return 0;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    BatchedSyevjArgs args{plan->d_order, plan->d_n, plan->d_aoff, plan->d_woff, A, W, V,
                          sweeps,        tol,       max_sweeps,   sort ? 1 : 0};
    return syevj_run(plan, args, st);
}

NMX_API int nmx_syevj_plan_autotune(nmx_ctx ctx, nmx_syevj_plan plan, const float *A, float *W,
                                    float *V, int32_t *sweeps, double tol, int max_sweeps,
                                    int sort, int reps, void *stream) {
    using namespace nmx;
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(plan != nullptr, 2, "plan is NULL");
    NMX_ARG_CHECK(A != nullptr || plan->count == 0, 3, "A is NULL");
    NMX_ARG_CHECK(W != nullptr || plan->count == 0, 4, "W is NULL");
    NMX_ARG_CHECK(V != nullptr || plan->count == 0, 5, "V is NULL");
    NMX_ARG_CHECK(tol >= 0.0, 7, "tol must be >= 0");
    NMX_ARG_CHECK(max_sweeps >= 0 && max_sweeps <= 1000, 8, "max_sweeps must be in 0..1000");
    NMX_ARG_CHECK(reps >= 1 && reps <= 100, 10, "reps must be in 1..100");
    if (plan->count == 0) return 0;
    DeviceGuard g(ctx->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    BatchedSyevjArgs args{plan->d_order, plan->d_n, plan->d_aoff, plan->d_woff, A, W, V,
                          sweeps,        tol,       max_sweeps,   sort ? 1 : 0};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    NMX_CUDA_TRY(cudaEventCreate(&e0));
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        set_error("autotune: event creation failed");
        return NMX_ERR_CUDA;
    }
    int rc = 0;
    for (size_t bi = 0; bi < plan->buckets.size() && !rc; ++bi) {
        auto best = plan->buckets[bi];
        float best_ms = 3.4e38f;
        for (const auto &shape : kSyevjShapes) {
            auto cand = plan->buckets[bi];
            if (syevj_configure_shape(ctx, cand, shape[0], shape[1]) != 0) {
                clear_error();  // a shape that does not fit is skipped
                continue;
            }
            float ms = 3.4e38f;
            for (int r = 0; r < reps && !rc; ++r) {
                if (cudaMemsetAsync(plan->d_counters + bi, 0, sizeof(int32_t), st) != cudaSuccess ||
                    cudaEventRecord(e0, st) != cudaSuccess) {
                    set_error("autotune: %s", cudaGetErrorString(cudaGetLastError()));
                    rc = NMX_ERR_CUDA;
                    break;
                }
                rc = syevj_launch(args, cand, plan->d_counters + bi, st);
                float t = 0.f;
                if (!rc && (cudaEventRecord(e1, st) != cudaSuccess ||
                            cudaEventSynchronize(e1) != cudaSuccess ||
                            cudaEventElapsedTime(&t, e0, e1) != cudaSuccess)) {
                    set_error("autotune: %s", cudaGetErrorString(cudaGetLastError()));
                    rc = NMX_ERR_CUDA;
                }
                ms = std::min(ms, t);
            }
            if (rc) break;
            if (ms < best_ms) {
                best_ms = ms;
                best = cand;
            }
        }
        plan->buckets[bi] = best;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (plan->graph) {
        cudaGraphExecDestroy(plan->graph);
        plan->graph = nullptr;
    }
    if (rc) return rc;
    // The last timed runs may have used other shapes: leave the outputs of
    // the kept schedule.
    return syevj_run(plan, args, st);
}

NMX_API int nmx_syevj_plan_schedule(nmx_syevj_plan plan, int32_t *nmax, int32_t *threads,
                                    int32_t *group, int32_t *ctas, int max_buckets,
                                    int32_t *nbuckets) {
    NMX_ARG_CHECK(plan != nullptr, 1, "plan is NULL");
    NMX_ARG_CHECK(max_buckets >= 0, 6, "max_buckets < 0");
    const int nb = (int)plan->buckets.size();
    for (int i = 0; i < nb && i < max_buckets; ++i) {
        if (nmax) nmax[i] = plan->buckets[i].nmax;
        if (threads) threads[i] = plan->buckets[i].threads;
        if (group) group[i] = plan->buckets[i].group;
        if (ctas) ctas[i] = plan->buckets[i].grid;
    }
    if (nbuckets) *nbuckets = nb;
    return 0;
}

NMX_API int nmx_syevj_batched_graph_f32(nmx_ctx ctx, nmx_syevj_plan plan, const float *A, float *W,
                                        float *V, int32_t *sweeps, double tol, int max_sweeps,
                                        int sort, void *stream) {
    using namespace nmx;
    NMX_ARG_CHECK(ctx != nullptr, 1, "ctx is NULL");
    NMX_ARG_CHECK(plan != nullptr, 2, "plan is NULL");
    NMX_ARG_CHECK(A != nullptr || plan->count == 0, 3, "A is NULL");
    NMX_ARG_CHECK(W != nullptr || plan->count == 0, 4, "W is NULL");
    NMX_ARG_CHECK(V != nullptr || plan->count == 0, 5, "V is NULL");
    NMX_ARG_CHECK(tol >= 0.0, 7, "tol must be >= 0");
    NMX_ARG_CHECK(max_sweeps >= 0 && max_sweeps <= 1000, 8, "max_sweeps must be in 0..1000");
    if (plan->count == 0) return 0;
    DeviceGuard g(ctx->device);
    const void *key[4] = {A, W, V, sweeps};
    if (!plan->graph || !std::equal(key, key + 4, plan->graph_key) || plan->graph_tol != tol ||
        plan->graph_max_sweeps != max_sweeps || plan->graph_sort != (sort ? 1 : 0)) {
        if (plan->graph) {
            cudaGraphExecDestroy(plan->graph);
            plan->graph = nullptr;
        }
        cudaStream_t cs = nullptr;
        NMX_CUDA_TRY(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
        cudaGraph_t graph = nullptr;
        int rc = 0;
        BatchedSyevjArgs args{plan->d_order, plan->d_n, plan->d_aoff, plan->d_woff, A, W, V,
                              sweeps,        tol,       max_sweeps,   sort ? 1 : 0};
        if (cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
            set_error("graph capture: %s", cudaGetErrorString(cudaGetLastError()));
            rc = NMX_ERR_CUDA;
        } else {
            rc = syevj_run(plan, args, cs);
            cudaError_t e = cudaStreamEndCapture(cs, &graph);
            if (!rc && e != cudaSuccess) {
                set_error("graph capture: %s", cudaGetErrorString(e));
                rc = NMX_ERR_CUDA;
            }
        }
        if (!rc && cudaGraphInstantiate(&plan->graph, graph, 0) != cudaSuccess) {
            set_error("graph instantiate: %s", cudaGetErrorString(cudaGetLastError()));
            plan->graph = nullptr;
            rc = NMX_ERR_CUDA;
        }
        if (graph) cudaGraphDestroy(graph);
        cudaStreamDestroy(cs);
        if (rc) return rc;
        std::copy(key, key + 4, plan->graph_key);
        plan->graph_tol = tol;
        plan->graph_max_sweeps = max_sweeps;
        plan->graph_sort = sort ? 1 : 0;
    }
    NMX_CUDA_TRY(cudaGraphLaunch(plan->graph, static_cast<cudaStream_t>(stream)));
    return 0;
}

}  // extern "C"
