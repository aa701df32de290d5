// runtime.cu - context, memory and launch orchestration behind the C ABI
// (include/g2_aimd.h).  Replaces PipelineExecutor (system/pipeline_executor.h:
// 44-207) and AppBase::initialize (system/appbase.h:93-114): instead of a
// host-synchronised BFS level loop with AIMD chunk retries, one persistent
// kernel pass per slab size is enqueued on a stream; roots that do not fit a
// warp's slab are deferred on the device to the next pass (bigger slab per
// warp), which replaces the overflow -> chunk/8 retry of
// system/subgraph_container.h:178-211 without host round trips.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "g2_aimd.h"
#include "g2_kernels.h"

struct g2_ctx {
    int device = 0;
    int sm_count = 148;
    uint64_t scratch_bytes = 0;
    // graph
    uint64_t *d_rp = nullptr;
    uint32_t *d_ci = nullptr;
    bool owns_csr = false;
    uint64_t n = 0, m = 0;
    uint32_t max_fwd = 0;  // max |N(v) ∩ (v, ∞)|
    uint32_t *d_fo = nullptr;  // forward-list offsets
    uint64_t fo_cap = 0;
    // work buffers
    uint32_t *d_scratch = nullptr;
    uint64_t scratch_words = 0;
    uint32_t *d_tasks = nullptr;   // root vertex per task (ordered)
    uint32_t *d_defer = nullptr;   // 3 deferred lists of tasks_cap each
    uint64_t tasks_cap = 0;
    uint64_t *d_root_nodes = nullptr;
    uint64_t root_nodes_cap = 0;
    unsigned long long *d_ctr = nullptr;  // [0..3] queue heads, [4..6] deferred counts
    int *d_status = nullptr;
    unsigned long long *d_out = nullptr;  // counters for the host entry points
    uint32_t out_cap = 0;
    // schedule
    uint64_t *d_keys = nullptr, *d_keys2 = nullptr;
    uint32_t *d_vals2 = nullptr;
    void *d_cub = nullptr;
    size_t cub_bytes = 0;
    uint64_t sched_cap = 0, sched2_cap = 0, scores_cap = 0;
    float *d_scores = nullptr;
    // plan
    g2::DevPlan plan{};
    bool has_plan = false;
    bool clique_plan = false;
    // diagnostics
    std::string cuda_err;
    uint64_t launches = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // around the three passes
    bool timed = false;
    unsigned long long *d_work = nullptr;
    cudaStream_t last_stream = nullptr;
};

namespace {

const char *kVersion = "g2aimd-b200 0.1 (sm_100a)";

int fail_cuda(g2_ctx *c, cudaError_t e, const char *where) {
    if (c) c->cuda_err = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? G2_ERR_OOM : G2_ERR_CUDA;
}

#define G2_TRY(call)                                          \
    do {                                                      \
        cudaError_t _e = (call);                              \
        if (_e != cudaSuccess) return fail_cuda(ctx, _e, #call); \
    } while (0)

template <class T>
int grow(g2_ctx *ctx, T *&p, uint64_t &cap, uint64_t need, const char *what) {
    if (need <= cap && p) return G2_OK;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc(&p, sizeof(T) * (need ? need : 1));
    if (e != cudaSuccess) return fail_cuda(ctx, e, what);
    cap = need;
    return G2_OK;
}

// fo[v] = offset in N(v) of the first neighbour larger than v (forward list
// start); out = max forward degree.
__global__ void forward_offsets_kernel(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint32_t *fo,
                                       unsigned int *out) {
    unsigned int best = 0;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t lo = rp[v], hi = rp[v + 1];
        uint64_t a = lo, b = hi;
        while (a < b) {
            uint64_t mid = a + ((b - a) >> 1);
            if (ci[mid] <= (uint32_t)v) a = mid + 1;
            else b = mid;
        }
        fo[v] = (uint32_t)(a - lo);
        unsigned int f = (unsigned int)(hi - a);
        best = f > best ? f : best;
    }
    for (int o = 16; o > 0; o >>= 1) {
        unsigned int y = __shfl_xor_sync(0xffffffffu, best, o);
        best = y > best ? y : best;
    }
    if ((threadIdx.x & 31) == 0) atomicMax(out, best);
}

__global__ void iota_kernel(uint32_t *t, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        t[i] = (uint32_t)i;
}

// Heuristic root cost: p * (p + |X0|) bitmap-row words of the root's local
// graph, a proxy of its set-up and search work; descending order = largest first.
__global__ void heuristic_keys_kernel(const uint64_t *rp, const uint32_t *ci, const uint32_t *src, uint64_t n,
                                      uint64_t *keys) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t v = src[i];
        uint64_t lo = rp[v], hi = rp[v + 1], a = lo, b = hi;
        while (a < b) {
            uint64_t mid = a + ((b - a) >> 1);
            if (ci[mid] <= v) a = mid + 1;
            else b = mid;
        }
        uint64_t p = hi - a, d = hi - lo;
        uint64_t cost = p * (p + d);
        keys[i] = ~cost;  // ascending sort of ~cost = descending cost
    }
}

__global__ void score_keys_kernel(const float *scores, uint64_t n, uint64_t *keys) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t b = __float_as_uint(scores[i]);
        b = (b & 0x80000000u) ? ~b : (b | 0x80000000u);  // order-preserving float -> uint
        keys[i] = ~(uint64_t)b;                           // descending score
    }
}

int default_warps(const g2_opts *o) { return (o && o->warps_per_block) ? (int)o->warps_per_block : 8; }

int default_blocks(g2_ctx *ctx, const g2_opts *o, int wpb) {
    if (o && o->blocks) return (int)o->blocks;
    // persistent grid: resident CTAs per SM x SMs
    int per_sm = std::max(1, 32 / wpb);
    return ctx->sm_count * per_sm;
}

// Upload / order the task list: d_tasks[i] = root of task i.
int prepare_tasks(g2_ctx *ctx, const uint32_t *sources, uint64_t nsrc, bool on_device, const g2_opts *o,
                  cudaStream_t st, std::vector<uint32_t> *order_out) {
    if (!sources) nsrc = ctx->n;
    uint64_t cap = ctx->tasks_cap;
    int rc = grow(ctx, ctx->d_tasks, cap, nsrc, "tasks");
    if (rc) return rc;
    if (cap != ctx->tasks_cap || !ctx->d_defer) {
        // three deferred-task lists with stride tasks_cap
        if (ctx->d_defer) cudaFree(ctx->d_defer);
        ctx->d_defer = nullptr;
        G2_TRY(cudaMalloc(&ctx->d_defer, sizeof(uint32_t) * 3 * std::max<uint64_t>(cap, 1)));
    }
    ctx->tasks_cap = cap;
    if (!sources) {
        iota_kernel<<<ctx->sm_count * 4, 256, 0, st>>>(ctx->d_tasks, nsrc);
        ctx->launches++;
    } else if (on_device) {
        G2_TRY(cudaMemcpyAsync(ctx->d_tasks, sources, sizeof(uint32_t) * nsrc, cudaMemcpyDeviceToDevice, st));
    } else {
        G2_TRY(cudaMemcpyAsync(ctx->d_tasks, sources, sizeof(uint32_t) * nsrc, cudaMemcpyHostToDevice, st));
    }
    uint32_t sched = o ? o->schedule : G2_SCHED_GIVEN;
    if (sched == G2_SCHED_GIVEN || nsrc < 2) return G2_OK;
    if (sched == G2_SCHED_SCORES && !(o && o->scores)) return G2_ERR_INVALID;
    // keys -> sort (task order) ; the permutation is kept for per-root outputs
    rc = grow(ctx, ctx->d_keys, ctx->sched_cap, nsrc, "keys");
    if (rc) return rc;
    uint64_t c2 = ctx->sched2_cap, c3 = ctx->sched2_cap;
    rc = grow(ctx, ctx->d_keys2, c2, nsrc, "keys2");
    if (!rc) rc = grow(ctx, ctx->d_vals2, c3, nsrc, "vals2");
    ctx->sched2_cap = std::min(c2, c3);
    if (rc) return rc;
    if (sched == G2_SCHED_HEURISTIC) {
        heuristic_keys_kernel<<<ctx->sm_count * 4, 256, 0, st>>>(ctx->d_rp, ctx->d_ci, ctx->d_tasks, nsrc,
                                                                ctx->d_keys);
    } else {
        rc = grow(ctx, ctx->d_scores, ctx->scores_cap, nsrc, "scores");
        if (rc) return rc;
        G2_TRY(cudaMemcpyAsync(ctx->d_scores, o->scores, sizeof(float) * nsrc, cudaMemcpyHostToDevice, st));
        score_keys_kernel<<<ctx->sm_count * 4, 256, 0, st>>>(ctx->d_scores, nsrc, ctx->d_keys);
    }
    ctx->launches++;
    size_t need = 0;
    cub::DeviceRadixSort::SortPairs(nullptr, need, ctx->d_keys, ctx->d_keys2, ctx->d_tasks, ctx->d_vals2,
                                    (int)nsrc, 0, 64, st);
    if (need > ctx->cub_bytes) {
        if (ctx->d_cub) cudaFree(ctx->d_cub);
        ctx->d_cub = nullptr;
        G2_TRY(cudaMalloc(&ctx->d_cub, need));
        ctx->cub_bytes = need;
    }
    G2_TRY(cub::DeviceRadixSort::SortPairs(ctx->d_cub, need, ctx->d_keys, ctx->d_keys2, ctx->d_tasks,
                                           ctx->d_vals2, (int)nsrc, 0, 64, st));
    ctx->launches += 4;
    G2_TRY(cudaMemcpyAsync(ctx->d_tasks, ctx->d_vals2, sizeof(uint32_t) * nsrc, cudaMemcpyDeviceToDevice, st));
    if (order_out) {
        order_out->resize(nsrc);
        G2_TRY(cudaMemcpyAsync(order_out->data(), ctx->d_tasks, sizeof(uint32_t) * nsrc, cudaMemcpyDeviceToHost,
                               st));
    }
    return G2_OK;
}

int ensure_scratch(g2_ctx *ctx) {
    if (ctx->d_scratch) return G2_OK;
    uint64_t words = ctx->scratch_bytes / 4;
    words &= ~63ull;
    G2_TRY(cudaMalloc(&ctx->d_scratch, words * 4));
    ctx->scratch_words = words;
    return G2_OK;
}

int ensure_counters(g2_ctx *ctx) {
    if (!ctx->d_ctr) G2_TRY(cudaMalloc(&ctx->d_ctr, sizeof(unsigned long long) * 16));
    if (!ctx->d_status) G2_TRY(cudaMalloc(&ctx->d_status, sizeof(int)));
    return G2_OK;
}

int status_to_code(int st) {
    if (st & g2::kStatusDeferOverflow) return G2_ERR_OVERFLOW;
    if (st & g2::kStatusStackOverflow) return G2_ERR_OVERFLOW;
    if (st & g2::kStatusBadPlan) return G2_ERR_INVALID;
    if (st & g2::kStatusHistOverflow) return G2_ERR_HIST;
    return G2_OK;
}

// Events for pass timing and the device work counter, as the flags ask.
int prepare_flags(g2_ctx *ctx, uint32_t flags, cudaStream_t st) {
    ctx->timed = (flags & G2_FLAG_TIME_KERNELS) != 0;
    ctx->last_stream = st;
    if (ctx->timed && !ctx->ev[0])
        for (auto &e : ctx->ev) G2_TRY(cudaEventCreate(&e));
    if (flags & G2_FLAG_WORK_MODEL) {
        if (!ctx->d_work) G2_TRY(cudaMalloc(&ctx->d_work, sizeof(unsigned long long)));
        G2_TRY(cudaMemsetAsync(ctx->d_work, 0, sizeof(unsigned long long), st));
    }
    return G2_OK;
}

int wpl_for(uint32_t p) {
    uint32_t W = (p + 31) / 32;
    return W <= 32 ? 1 : W <= 64 ? 2 : W <= 128 ? 4 : 8;
}

// Enqueue the MCE passes; counters land in d_out.
int mce_enqueue(g2_ctx *ctx, uint64_t ntasks, const g2_opts *o, unsigned long long *d_out, uint32_t hist_len,
                uint64_t *d_root_nodes, cudaStream_t st) {
    int rc = ensure_scratch(ctx);
    if (rc) return rc;
    rc = ensure_counters(ctx);
    if (rc) return rc;
    if (ctx->max_fwd > 32u * 32u * 8u) return G2_ERR_UNSUPPORTED;
    G2_TRY(cudaMemsetAsync(ctx->d_ctr, 0, sizeof(unsigned long long) * 16, st));
    G2_TRY(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), st));
    G2_TRY(cudaMemsetAsync(d_out, 0, sizeof(unsigned long long) * (1 + hist_len), st));
    const uint32_t flags = o ? o->flags : 0u;
    rc = prepare_flags(ctx, flags, st);
    if (rc) return rc;
    const int wpb = default_warps(o);
    const int blocks = default_blocks(ctx, o, wpb);
    // pass 1: every task, WPL=1, one slab per resident warp
    // pass 2: deferred roots, 2 warps per SM, WPL for the widest root
    // pass 3: what is still deferred, one warp owning the whole slab
    struct Pass {
        int blocks, wpb, wpl;
    } passes[3] = {{blocks, wpb, 1}, {ctx->sm_count, 2, wpl_for(ctx->max_fwd)}, {1, 1, wpl_for(ctx->max_fwd)}};
    for (int k = 0; k < 3; k++) {
        g2::MceArgs a{};
        a.rp = ctx->d_rp;
        a.ci = ctx->d_ci;
        a.fo = ctx->d_fo;
        a.tasks = ctx->d_tasks;
        a.task_index = k == 0 ? nullptr : ctx->d_defer + (uint64_t)(k - 1) * ctx->tasks_cap;
        a.ntasks = k == 0 ? ntasks : 0;
        a.ntasks_dev = k == 0 ? nullptr : ctx->d_ctr + 4 + (k - 1);
        a.head = ctx->d_ctr + k;
        a.chunk = k == 0 ? 2 : 1;
        a.hist_len = hist_len;
        a.scratch = ctx->d_scratch;
        uint64_t nw = (uint64_t)passes[k].blocks * passes[k].wpb;
        a.words_per_warp = (ctx->scratch_words / nw) & ~63ull;
        a.out = d_out;
        a.deferred = ctx->d_defer + (uint64_t)k * ctx->tasks_cap;
        a.ndeferred = ctx->d_ctr + 4 + k;
        a.deferred_cap = ctx->tasks_cap;
        a.root_nodes = d_root_nodes;
        a.status = ctx->d_status;
        a.final_pass = k == 2;
        a.work = (flags & G2_FLAG_WORK_MODEL) ? ctx->d_work : nullptr;
        if (ctx->timed && k == 0) G2_TRY(cudaEventRecord(ctx->ev[0], st));
        cudaError_t e = g2::mce_launch(passes[k].wpl, a, passes[k].blocks, passes[k].wpb, st);
        if (e != cudaSuccess) return fail_cuda(ctx, e, "mce_launch");
        if (ctx->timed) G2_TRY(cudaEventRecord(ctx->ev[k + 1], st));
        ctx->launches++;
    }
    return G2_OK;
}

}  // namespace

extern "C" {

const char *g2_version(void) { return kVersion; }

const char *g2_strerror(int code) {
    switch (code) {
        case G2_OK: return "ok";
        case G2_ERR_INVALID: return "invalid argument";
        case G2_ERR_CUDA: return "CUDA runtime error";
        case G2_ERR_OOM: return "out of memory";
        case G2_ERR_TIMEOUT: return "bounded device wait expired";
        case G2_ERR_OVERFLOW: return "scratch and spill capacity exhausted";
        case G2_ERR_NO_GRAPH: return "no graph loaded";
        case G2_ERR_NO_PLAN: return "no query plan set";
        case G2_ERR_UNSUPPORTED: return "unsupported size";
        case G2_ERR_IO: return "I/O error";
        case G2_ERR_HIST: return "clique larger than the histogram";
        default: return "unknown error";
    }
}

const char *g2_last_cuda_error(const g2_ctx *ctx) { return ctx ? ctx->cuda_err.c_str() : ""; }

uint64_t g2_last_launch_count(const g2_ctx *ctx) { return ctx ? ctx->launches : 0; }

int g2_pass_time_ms(g2_ctx *ctx, int pass, float *ms) {
    if (!ctx || !ms || pass < 0 || pass > 2 || !ctx->timed) return G2_ERR_INVALID;
    G2_TRY(cudaEventSynchronize(ctx->ev[pass + 1]));
    G2_TRY(cudaEventElapsedTime(ms, ctx->ev[pass], ctx->ev[pass + 1]));
    return G2_OK;
}

int g2_last_work_bytes(g2_ctx *ctx, uint64_t *bytes) {
    if (!ctx || !bytes || !ctx->d_work) return G2_ERR_INVALID;
    unsigned long long h = 0;
    G2_TRY(cudaStreamSynchronize(ctx->last_stream));
    G2_TRY(cudaMemcpy(&h, ctx->d_work, sizeof(h), cudaMemcpyDeviceToHost));
    *bytes = h;
    return G2_OK;
}

int g2_open(int device, uint64_t scratch_bytes, g2_ctx **out) {
    if (!out) return G2_ERR_INVALID;
    *out = nullptr;
    int ndev = 0;
    g2_ctx *ctx = nullptr;
    G2_TRY(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) return G2_ERR_INVALID;
    ctx = new g2_ctx();
    ctx->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) {
        delete ctx;
        return fail_cuda(nullptr, e, "g2_open");
    }
    ctx->scratch_bytes = scratch_bytes ? scratch_bytes : (4ull << 30);
    *out = ctx;
    return G2_OK;
}

int g2_close(g2_ctx *ctx) {
    if (!ctx) return G2_ERR_INVALID;
    cudaSetDevice(ctx->device);
    if (ctx->owns_csr) {
        cudaFree(ctx->d_rp);
        cudaFree(ctx->d_ci);
    }
    void *bufs[] = {ctx->d_fo, ctx->d_scratch, ctx->d_tasks, ctx->d_defer, ctx->d_root_nodes, ctx->d_ctr, ctx->d_status,
                    ctx->d_out, ctx->d_keys, ctx->d_keys2, ctx->d_vals2, ctx->d_cub, ctx->d_scores};
    for (void *b : bufs)
        if (b) cudaFree(b);
    if (ctx->d_work) cudaFree(ctx->d_work);
    for (auto &e : ctx->ev)
        if (e) cudaEventDestroy(e);
    delete ctx;
    return G2_OK;
}

static int after_load(g2_ctx *ctx) {
    int rc = grow(ctx, ctx->d_fo, ctx->fo_cap, std::max<uint64_t>(ctx->n, 1), "forward offsets");
    if (rc) return rc;
    unsigned int *d_max = nullptr;
    G2_TRY(cudaMalloc(&d_max, sizeof(unsigned int)));
    G2_TRY(cudaMemset(d_max, 0, sizeof(unsigned int)));
    if (ctx->n) forward_offsets_kernel<<<ctx->sm_count * 4, 256>>>(ctx->d_rp, ctx->d_ci, ctx->n, ctx->d_fo, d_max);
    ctx->launches++;
    unsigned int h = 0;
    cudaError_t e = cudaMemcpy(&h, d_max, sizeof(unsigned int), cudaMemcpyDeviceToHost);
    cudaFree(d_max);
    if (e != cudaSuccess) return fail_cuda(ctx, e, "fwd_max");
    ctx->max_fwd = h;
    return G2_OK;
}

int g2_load_csr(g2_ctx *ctx, const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n, uint64_t m) {
    if (!ctx || !row_ptrs || (!cols && m) || n >= (1ull << 32)) return G2_ERR_INVALID;
    if (row_ptrs[n] != m) return G2_ERR_INVALID;
    G2_TRY(cudaSetDevice(ctx->device));
    if (ctx->owns_csr) {
        cudaFree(ctx->d_rp);
        cudaFree(ctx->d_ci);
    }
    ctx->d_rp = nullptr;
    ctx->d_ci = nullptr;
    ctx->owns_csr = true;
    G2_TRY(cudaMalloc(&ctx->d_rp, sizeof(uint64_t) * (n + 1)));
    G2_TRY(cudaMalloc(&ctx->d_ci, sizeof(uint32_t) * (m ? m : 1)));
    G2_TRY(cudaMemcpy(ctx->d_rp, row_ptrs, sizeof(uint64_t) * (n + 1), cudaMemcpyHostToDevice));
    if (m) G2_TRY(cudaMemcpy(ctx->d_ci, cols, sizeof(uint32_t) * m, cudaMemcpyHostToDevice));
    ctx->n = n;
    ctx->m = m;
    return after_load(ctx);
}

int g2_load_csr_device(g2_ctx *ctx, const uint64_t *d_row_ptrs, const uint32_t *d_cols, uint64_t n, uint64_t m) {
    if (!ctx || !d_row_ptrs || (!d_cols && m) || n >= (1ull << 32)) return G2_ERR_INVALID;
    G2_TRY(cudaSetDevice(ctx->device));
    if (ctx->owns_csr) {
        cudaFree(ctx->d_rp);
        cudaFree(ctx->d_ci);
    }
    ctx->d_rp = const_cast<uint64_t *>(d_row_ptrs);
    ctx->d_ci = const_cast<uint32_t *>(d_cols);
    ctx->owns_csr = false;
    ctx->n = n;
    ctx->m = m;
    return after_load(ctx);
}

int g2_set_plan(g2_ctx *ctx, const g2_plan *p) {
    if (!ctx || !p) return G2_ERR_INVALID;
    const uint32_t k = p->k;
    if (k < 2 || k > G2_MAX_QUERY) return G2_ERR_UNSUPPORTED;
    g2::DevPlan d{};
    d.k = k;
    for (uint32_t u = 0; u < k; u++)
        if (p->order[u] >= k || p->id2order[p->order[u]] != u) return G2_ERR_INVALID;
    bool clique = true;
    for (uint32_t i = 0; i < k; i++) {
        const uint32_t u = p->order[i];  // query vertex at position i
        if (i > 0 && p->bn_count[i] == 0) return G2_ERR_INVALID;
        d.bn_count[i] = p->bn_count[i];
        for (uint32_t j = 0; j < p->bn_count[i]; j++) {
            uint32_t pos = p->id2order[p->bn[i][j]];
            if (pos >= i) return G2_ERR_INVALID;
            d.bn_pos[i][j] = pos;
        }
        d.cond_count[i] = p->cond_count[u];
        uint32_t larger = 0;
        for (uint32_t j = 0; j < p->cond_count[u]; j++) {
            uint32_t pos = p->id2order[p->cond[u][j][1]];
            if (pos >= i || p->cond[u][j][0] > G2_COND_NON_EQUAL) return G2_ERR_INVALID;
            d.cond_op[i][j] = p->cond[u][j][0];
            d.cond_pos[i][j] = pos;
            larger += p->cond[u][j][0] == G2_COND_LARGER_THAN;
        }
        if (i > 0 && (p->bn_count[i] != i || larger != i)) clique = false;
        d.share[i] = p->share[i];
    }
    d.clique = clique ? 1u : 0u;
    ctx->plan = d;
    ctx->has_plan = true;
    ctx->clique_plan = clique;
    return G2_OK;
}

int g2_mce_run_device(g2_ctx *ctx, const uint32_t *d_sources, uint64_t nsrc, const g2_opts *opts, uint64_t *d_out,
                      uint32_t hist_len, void *stream) {
    if (!ctx || !d_out) return G2_ERR_INVALID;
    if (!ctx->d_rp) return G2_ERR_NO_GRAPH;
    G2_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    ctx->launches = 0;
    int rc = prepare_tasks(ctx, d_sources, nsrc, true, opts, st, nullptr);
    if (rc) return rc;
    if (!d_sources) nsrc = ctx->n;
    return mce_enqueue(ctx, nsrc, opts, reinterpret_cast<unsigned long long *>(d_out), hist_len, nullptr, st);
}

int g2_mce_run(g2_ctx *ctx, const uint32_t *sources, uint64_t nsrc, const g2_opts *opts, uint64_t *count,
               uint64_t *hist, uint32_t hist_len) {
    if (!ctx || !count || (hist && hist_len == 0)) return G2_ERR_INVALID;
    if (!ctx->d_rp) return G2_ERR_NO_GRAPH;
    G2_TRY(cudaSetDevice(ctx->device));
    ctx->launches = 0;
    const uint32_t hl = hist ? hist_len : 1u;
    cudaStream_t st = nullptr;
    std::vector<uint32_t> order;
    const bool want_nodes = opts && opts->root_nodes;
    int rc = prepare_tasks(ctx, sources, nsrc, false, opts, st, want_nodes ? &order : nullptr);
    if (rc) return rc;
    if (!sources) nsrc = ctx->n;
    uint64_t rncap = ctx->root_nodes_cap;
    if (want_nodes) {
        rc = grow(ctx, ctx->d_root_nodes, rncap, nsrc, "root_nodes");
        ctx->root_nodes_cap = rncap;
        if (rc) return rc;
    }
    uint64_t oc = ctx->out_cap;
    rc = grow(ctx, ctx->d_out, oc, 1 + hl, "out");
    ctx->out_cap = (uint32_t)oc;
    if (rc) return rc;
    g2_opts o2{};
    if (opts) o2 = *opts;
    if (o2.work_bytes) o2.flags |= G2_FLAG_WORK_MODEL;
    rc = mce_enqueue(ctx, nsrc, &o2, ctx->d_out, hl, want_nodes ? ctx->d_root_nodes : nullptr, st);
    if (rc) return rc;
    std::vector<unsigned long long> h(1 + hl);
    int status = 0;
    G2_TRY(cudaMemcpy(h.data(), ctx->d_out, sizeof(unsigned long long) * (1 + hl), cudaMemcpyDeviceToHost));
    G2_TRY(cudaMemcpy(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    unsigned long long ndef3 = 0;
    G2_TRY(cudaMemcpy(&ndef3, ctx->d_ctr + 6, sizeof(unsigned long long), cudaMemcpyDeviceToHost));
    if (ndef3) return G2_ERR_OVERFLOW;
    *count = h[0];
    if (hist)
        for (uint32_t s = 0; s < hist_len; s++) hist[s] = h[1 + s];
    if (o2.work_bytes) {
        rc = g2_last_work_bytes(ctx, o2.work_bytes);
        if (rc) return rc;
    }
    if (want_nodes) {
        std::vector<uint64_t> rn(nsrc);
        G2_TRY(cudaMemcpy(rn.data(), ctx->d_root_nodes, sizeof(uint64_t) * nsrc, cudaMemcpyDeviceToHost));
        if (!order.empty()) {
            // task i ran root order[i]; map back to the caller's source index
            std::vector<uint64_t> pos_of(ctx->n, ~0ull);
            if (sources)
                for (uint64_t i = 0; i < nsrc; i++) pos_of[sources[i]] = i;
            for (uint64_t i = 0; i < nsrc; i++) {
                uint64_t j = sources ? pos_of[order[i]] : order[i];
                opts->root_nodes[j] = rn[i];
            }
        } else {
            memcpy(opts->root_nodes, rn.data(), sizeof(uint64_t) * nsrc);
        }
    }
    return status_to_code(status);
}

int g2_match_run_device(g2_ctx *ctx, const uint32_t *d_sources, uint64_t nsrc, const g2_opts *opts,
                        uint64_t *d_out, void *stream) {
    if (!ctx || !d_out) return G2_ERR_INVALID;
    if (!ctx->d_rp) return G2_ERR_NO_GRAPH;
    if (!ctx->has_plan) return G2_ERR_NO_PLAN;
    G2_TRY(cudaSetDevice(ctx->device));
    cudaStream_t st = (cudaStream_t)stream;
    ctx->launches = 0;
    int rc = prepare_tasks(ctx, d_sources, nsrc, true, opts, st, nullptr);
    if (rc) return rc;
    if (!d_sources) nsrc = ctx->n;
    rc = ensure_scratch(ctx);
    if (rc) return rc;
    rc = ensure_counters(ctx);
    if (rc) return rc;
    G2_TRY(cudaMemsetAsync(ctx->d_ctr, 0, sizeof(unsigned long long) * 16, st));
    G2_TRY(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), st));
    G2_TRY(cudaMemsetAsync(d_out, 0, sizeof(unsigned long long), st));
    const uint32_t flags = opts ? opts->flags : 0u;
    rc = prepare_flags(ctx, flags, st);
    if (rc) return rc;
    int wpl = wpl_for(ctx->max_fwd);
    int wpb = default_warps(opts);
    while (wpb > 1 && g2::match_smem_bytes(wpl, wpb) > 200 * 1024) wpb /= 2;
    const int blocks = default_blocks(ctx, opts, wpb);
    g2::MatchArgs a{};
    a.rp = ctx->d_rp;
    a.ci = ctx->d_ci;
    a.fo = ctx->d_fo;
    a.tasks = ctx->d_tasks;
    a.ntasks = nsrc;
    a.head = ctx->d_ctr;
    a.chunk = 4;
    a.scratch = ctx->d_scratch;
    a.words_per_warp = (ctx->scratch_words / ((uint64_t)blocks * wpb)) & ~63ull;
    if (a.words_per_warp / (ctx->plan.k > 2 ? ctx->plan.k - 2 : 1) < 64) return G2_ERR_OVERFLOW;
    a.out = reinterpret_cast<unsigned long long *>(d_out);
    a.root_nodes = nullptr;
    a.status = ctx->d_status;
    a.work = (flags & G2_FLAG_WORK_MODEL) ? ctx->d_work : nullptr;
    const bool clique = ctx->clique_plan && !(opts && opts->intersect_mode == 1);
    if (ctx->timed) G2_TRY(cudaEventRecord(ctx->ev[0], st));
    cudaError_t e = g2::match_launch(ctx->plan, a, blocks, wpb, st, clique, wpl);
    if (e != cudaSuccess) return fail_cuda(ctx, e, "match_launch");
    if (ctx->timed) G2_TRY(cudaEventRecord(ctx->ev[1], st));
    ctx->launches++;
    return G2_OK;
}

int g2_match_run(g2_ctx *ctx, const uint32_t *sources, uint64_t nsrc, const g2_opts *opts, uint64_t *count) {
    if (!ctx || !count) return G2_ERR_INVALID;
    if (!ctx->d_rp) return G2_ERR_NO_GRAPH;
    if (!ctx->has_plan) return G2_ERR_NO_PLAN;
    G2_TRY(cudaSetDevice(ctx->device));
    uint32_t *d_src = nullptr;
    if (sources) {
        G2_TRY(cudaMalloc(&d_src, sizeof(uint32_t) * std::max<uint64_t>(nsrc, 1)));
        cudaError_t e = cudaMemcpy(d_src, sources, sizeof(uint32_t) * nsrc, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(d_src);
            return fail_cuda(ctx, e, "sources");
        }
    }
    uint64_t oc = ctx->out_cap;
    int rc = grow(ctx, ctx->d_out, oc, 1, "out");
    ctx->out_cap = (uint32_t)oc;
    g2_opts o2{};
    if (opts) o2 = *opts;
    if (o2.work_bytes) o2.flags |= G2_FLAG_WORK_MODEL;
    if (!rc) rc = g2_match_run_device(ctx, sources ? d_src : nullptr, nsrc, &o2, (uint64_t *)ctx->d_out, nullptr);
    if (!rc && o2.work_bytes) rc = g2_last_work_bytes(ctx, o2.work_bytes);
    unsigned long long h = 0;
    int status = 0;
    if (!rc) {
        cudaError_t e = cudaMemcpy(&h, ctx->d_out, sizeof(h), cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost);
        if (e != cudaSuccess) rc = fail_cuda(ctx, e, "match result");
    }
    if (d_src) cudaFree(d_src);
    if (rc) return rc;
    *count = h;
    return status_to_code(status);
}

}  // extern "C"
