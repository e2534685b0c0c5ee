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

// Per-group shared-memory floats for matrices up to nmax.
__host__ __device__ inline int syevj_group_floats(int nmax) {
    int ld = nmax | 1;
    // A, V, then rotations (c, s as float2 pairs of doubles -> 4 floats) and
    // index pairs (2 ints), and a float64 reduction scratch.
    return 2 * nmax * ld + (nmax / 2 + 1) * 4 + (nmax / 2 + 1) * 2 + 2 * 64;
}

template <int G>
__device__ void syevj_one(const BatchedSyevjArgs &args, int mi, float *As, float *Vs, double *cs,
                          int *pq, double *red, int gt) {
    const int n = args.ns[mi];
    const int ld = n | 1;
    const int m = n + (n & 1);
    const int half = m / 2;
    const float *A = args.A + args.a_off[mi];
    float *V = args.V + args.a_off[mi];
    float *W = args.W + args.w_off[mi];

    for (int e = gt; e < n * n; e += G) {
        int i = e / n, j = e - i * n;
        As[i * ld + j] = A[e];
        Vs[i * ld + j] = i == j ? 1.f : 0.f;
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
            // Pairs and float64 rotations for this round.
            for (int k = gt; k < half; k += G) {
                int a = tourney(k, r, m), b = tourney(m - 1 - k, r, m);
                int p = min(a, b), q = max(a, b);
                double c = 1.0, s = 0.0;
                if (q < n) {
                    // numax's angle, evaluated with reciprocal square roots
                    // and one correctly rounded reciprocal (the chain of two
                    // square roots and two divisions is the round's latency).
                    double apq = As[p * ld + q], app = As[p * ld + p], aqq = As[q * ld + q];
                    double d = aqq - app;
                    double two = 2.0 * apq;
                    const double r2 = d * d + two * two;
                    const double radius = r2 > 0.0 ? r2 * rsqrt(r2) : 0.0;
                    double safe = guard_nonzero(fabs(d) + radius, 1e-30);
                    double t = copysign(1.0, d) * two * __drcp_rn(safe);
                    c = rsqrt(1.0 + t * t);
                    s = t * c;
                }
                cs[2 * k] = c;
                cs[2 * k + 1] = s;
                pq[2 * k] = p;
                pq[2 * k + 1] = q;
            }
            group_sync<G>();
            // 2x2 blocks: rows of pair kr, columns of pair kc.  The rotations
            // were formed in float64; they are applied to the float32 data in
            // float32.  Lane = column pair (half <= 32), warp = row pairs.
            {
                constexpr int NWG = G / 32;
                const int lane = gt & 31, wg = gt >> 5;
                const int kc = lane;
                const bool colok = kc < half;
                const int u = colok ? pq[2 * kc] : 0, v = colok ? pq[2 * kc + 1] : 0;
                const float cc = colok ? (float)cs[2 * kc] : 1.f;
                const float sc = colok ? (float)cs[2 * kc + 1] : 0.f;
                for (int kr = wg; kr < half; kr += NWG) {
                    if (!colok) continue;
                    const int p = pq[2 * kr], q = pq[2 * kr + 1];
                    if (q >= n && v >= n) continue;
                    const float cr = (float)cs[2 * kr], sr = (float)cs[2 * kr + 1];
                    if (q < n && v < n) {
                        const float b00 = As[p * ld + u], b01 = As[p * ld + v];
                        const float b10 = As[q * ld + u], b11 = As[q * ld + v];
                        // rows: [c -s; s c] applied from the left
                        const float r00 = cr * b00 - sr * b10, r01 = cr * b01 - sr * b11;
                        const float r10 = sr * b00 + cr * b10, r11 = sr * b01 + cr * b11;
                        // columns: [c s; -s c] applied from the right
                        float o00 = cc * r00 - sc * r01, o01 = sc * r00 + cc * r01;
                        float o10 = cc * r10 - sc * r11, o11 = sc * r10 + cc * r11;
                        if (kr == kc) {
                            o01 = 0.f;  // the annihilated pair
                            o10 = 0.f;
                        }
                        As[p * ld + u] = o00;
                        As[p * ld + v] = o01;
                        As[q * ld + u] = o10;
                        As[q * ld + v] = o11;
                    } else if (q < n) {  // column pair has the dummy index
                        const float b0 = As[p * ld + u], b1 = As[q * ld + u];
                        As[p * ld + u] = cr * b0 - sr * b1;
                        As[q * ld + u] = sr * b0 + cr * b1;
                    } else {  // row pair has the dummy index
                        const float b0 = As[p * ld + u], b1 = As[p * ld + v];
                        As[p * ld + u] = cc * b0 - sc * b1;
                        As[p * ld + v] = sc * b0 + cc * b1;
                    }
                }
                // V := V J: warp = rows of V, lane = column pair.
                if (colok && v < n)
                    for (int i = wg; i < n; i += NWG) {
                        const float vp = Vs[i * ld + u], vq = Vs[i * ld + v];
                        Vs[i * ld + u] = cc * vp - sc * vq;
                        Vs[i * ld + v] = sc * vp + cc * vq;
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
    const int ld = nmax | 1;
    const int per_group = syevj_group_floats(nmax);
    float *base = reinterpret_cast<float *>(smem_raw) + (size_t)g * ((per_group + 3) & ~3);
    float *As = base;
    float *Vs = As + nmax * ld;
    double *cs =
        reinterpret_cast<double *>((reinterpret_cast<uintptr_t>(Vs + nmax * ld) + 7) & ~uintptr_t(7));
    int *pq = reinterpret_cast<int *>(cs + 2 * (nmax / 2 + 1));
    double *red = reinterpret_cast<double *>(
        (reinterpret_cast<uintptr_t>(pq + 2 * (nmax / 2 + 1)) + 7) & ~uintptr_t(7));
    __shared__ int s_item[NG];
    for (;;) {
        if (gt == 0) s_item[g] = atomicAdd(counter, 1);
        group_sync<G>();
        const int item = begin + s_item[g];
        group_sync<G>();
        if (item >= end) break;
        syevj_one<G>(args, args.order[item], As, Vs, cs, pq, red, gt);
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
    NMX_CUDA_TRY(cudaMemsetAsync(plan->d_counters, 0, sizeof(int32_t) * plan->buckets.size(), st));
    for (size_t bi = 0; bi < plan->buckets.size(); ++bi) {
        const auto &b = plan->buckets[bi];
        if (b.group == 32)
            syevj_batched_kernel<128, 32><<<b.grid, 128, b.smem, st>>>(args, b.begin, b.end, b.nmax,
                                                                       plan->d_counters + bi);
        else
            syevj_batched_kernel<128, 128><<<b.grid, 128, b.smem, st>>>(args, b.begin, b.end, b.nmax,
                                                                        plan->d_counters + bi);
        NMX_CUDA_TRY(cudaGetLastError());
    }
    return 0;
}

}  // extern "C"
