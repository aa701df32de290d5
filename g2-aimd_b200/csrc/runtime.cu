// runtime.cu - context, memory and launch orchestration behind the C ABI
// (include/g2_aimd.h).  Replaces PipelineExecutor (system/pipeline_executor.h:
// 44-207) and AppBase::initialize (system/appbase.h:93-114): instead of a
// host-synchronised BFS level loop with AIMD chunk retries, one persistent
// kernel pass per slab size is enqueued on a stream; roots that do not fit a
// warp's slab are deferred on the device to the next pass (bigger slab per
// warp), which replaces the overflow -> chunk/8 retry of
// system/subgraph_container.h:178-211 without host round trips.  Task
// generation (root order, heavy-root splits, the learned cost model's
// inference) also runs on the device.
#include <cuda_runtime.h>

#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdlib>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <random>
#include <string>
#include <unordered_map>
#include <vector>

#include "g2_aimd.h"
#include "g2_kernels.h"
#include "runtime_internal.h"

namespace g2rt {

int fail_cuda(g2_ctx *c, cudaError_t e, const char *where) {
    if (c) c->cuda_err = std::string(where) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? G2_ERR_OOM : G2_ERR_CUDA;
}

int fail_cuda_if(g2_ctx *c, cudaError_t e, const char *where) { return e == cudaSuccess ? G2_OK : fail_cuda(c, e, where); }

}  // namespace g2rt

using namespace g2rt;

namespace {

const char *kVersion = "g2aimd-b200 0.2 (sm_100a)";

const uint32_t *core_of(const g2_ctx *ctx) { return ctx->core_loaded ? ctx->d_core : nullptr; }

int cub_space(g2_ctx *ctx, size_t need) {
    if (need <= ctx->cub_bytes && ctx->d_cub) return G2_OK;
    if (ctx->d_cub) cudaFree(ctx->d_cub);
    ctx->d_cub = nullptr;
    ctx->cub_bytes = 0;
    G2_TRY(cudaMalloc(&ctx->d_cub, need ? need : 16));
    ctx->cub_bytes = need;
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

// out[perm[v]] = in[v].
__global__ void rename_kernel(const uint32_t *in, const uint32_t *perm, uint64_t n, uint32_t *out) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        out[perm[v]] = in[v];
}

__global__ void iota_kernel(uint32_t *t, uint64_t n) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        t[i] = (uint32_t)i;
}

// Plain heuristic root cost: p * (p + deg) + 1 (bitmap-row words of the root's
// local graph, a proxy of its set-up and search work); total for the split target.
__global__ void heuristic_cost_kernel(const uint64_t *rp, const uint32_t *fo, const uint32_t *src, uint64_t n,
                                      float *cost, float *total) {
    float local = 0.f;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t v = src[i];
        const float d = (float)(rp[v + 1] - rp[v]), p = d - (float)fo[v];
        const float c = p * (p + d) + 1.f;
        cost[i] = c;
        local += c;
    }
    for (int o = 16; o > 0; o >>= 1) local += __shfl_xor_sync(0xffffffffu, local, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(total, local);
}

__device__ __forceinline__ uint32_t float_key(float c) {  // order-preserving float -> uint
    uint32_t b = __float_as_uint(c);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}

// One task per root: key = (descending cost, root slot).
__global__ void cost_keys_kernel(const float *cost, uint64_t n, uint64_t *keys) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        keys[i] = ((uint64_t)(~float_key(cost[i])) << 32) | (uint32_t)i;
}

// Tasks per root: ceil(cost / target) in 1..256, target = total * share.
__global__ void split_count_kernel(const float *cost, const float *total, uint64_t n, float share, uint32_t *S) {
    const float target = fmaxf(*total * share, 1.f);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const float k = ceilf(cost[i] / target);
        S[i] = (uint32_t)fminf(fmaxf(k, 1.f), 256.f);
    }
}

// Expand root i into S[i] tasks at off[i]; key = (descending per-task cost, slot).
__global__ void split_scatter_kernel(const uint32_t *src, const float *cost, const uint32_t *S, const uint32_t *off,
                                     uint64_t n, uint64_t cap, uint32_t *roots, uint32_t *parts, uint64_t *keys) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = S[i];
        const uint32_t kb = ~float_key(cost[i] / (float)s);
        for (uint32_t j = 0; j < s; j++) {
            const uint64_t t = (uint64_t)off[i] + j;
            if (t >= cap) break;
            roots[t] = src[i];
            parts[t] = (s << 16) | j;
            keys[t] = ((uint64_t)kb << 32) | (uint32_t)t;
        }
    }
}

__global__ void split_total_kernel(const uint32_t *S, const uint32_t *off, uint64_t n, uint64_t cap,
                                   unsigned long long *ntasks) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        unsigned long long t = n ? (unsigned long long)off[n - 1] + S[n - 1] : 0ull;
        *ntasks = t < cap ? t : cap;
    }
}

// tasks[i] = roots[slot of the i-th smallest key]; unused slots sort last.
__global__ void gather_tasks_kernel(const uint64_t *keys_sorted, const uint32_t *roots, const uint32_t *parts,
                                    uint64_t cap, uint32_t *tasks, uint32_t *task_part) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < cap; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t k = keys_sorted[i];
        if (k == ~0ull) {
            tasks[i] = 0;
            if (task_part) task_part[i] = 1u << 16;
            continue;
        }
        const uint32_t t = (uint32_t)(k & 0xffffffffull);
        tasks[i] = roots[t];
        if (task_part) task_part[i] = parts ? parts[t] : (1u << 16);
    }
}

// Per-graph sums of per-task counts: graph of a task's root by binary search
// over the batch's vertex offsets, partial sums in shared memory per CTA.
constexpr uint32_t kMaxBatchGraphs = 4096;
__global__ void segment_sum_kernel(const uint32_t *tasks, const uint64_t *per_task, uint64_t cap,
                                   const unsigned long long *ntask_dev, const uint64_t *goff, uint32_t ngraphs,
                                   unsigned long long *out) {
    __shared__ unsigned long long part[kMaxBatchGraphs];
    for (uint32_t g = threadIdx.x; g < ngraphs; g += blockDim.x) part[g] = 0ull;
    __syncthreads();
    const uint64_t n = ntask_dev ? (*ntask_dev < cap ? *ntask_dev : cap) : cap;
    for (uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t c = per_task[t];
        if (!c) continue;
        const uint64_t v = tasks[t];
        uint32_t lo = 0, hi = ngraphs;  // last g with goff[g] <= v
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (goff[mid] <= v) lo = mid;
            else hi = mid;
        }
        atomicAdd(part + lo, (unsigned long long)c);
    }
    __syncthreads();
    for (uint32_t g = threadIdx.x; g < ngraphs; g += blockDim.x)
        if (part[g]) atomicAdd(out + g, part[g]);
}

int default_warps(const g2_opts *o) { return (o && o->warps_per_block) ? (int)o->warps_per_block : 8; }

// Persistent grid: the CTAs that are resident at once (occupancy of the kernel
// the launch runs), so that no CTA waits for another to leave.
int default_blocks(g2_ctx *ctx, const g2_opts *o, int wpb, int resident_per_sm) {
    if (o && o->blocks) return (int)o->blocks;
    const int per_sm = resident_per_sm > 0 ? resident_per_sm : std::max(1, 32 / wpb);
    return ctx->sm_count * per_sm;
}

// Result of task generation.
int sort_keys(g2_ctx *ctx, uint64_t n, cudaStream_t st) {
    size_t need = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, need, ctx->d_keys, ctx->d_keys2, (int)n, 0, 64, st);
    int rc = cub_space(ctx, need);
    if (rc) return rc;
    G2_TRY(cub::DeviceRadixSort::SortKeys(ctx->d_cub, need, ctx->d_keys, ctx->d_keys2, (int)n, 0, 64, st));
    ctx->launches += 4;
    return G2_OK;
}

// Task generation: upload the roots, compute the schedule's cost per root (the
// learned model's features + MLP run here, in one kernel), optionally split
// heavy roots, sort the tasks by descending cost.  No host synchronisation.
}  // namespace

namespace g2rt {

int prepare_tasks(g2_ctx *ctx, const uint32_t *sources, uint64_t nsrc, bool on_device, const g2_opts *o,
                  uint64_t nwarps, cudaStream_t st, TaskList *tl, bool mce) {
    if (!sources) nsrc = ctx->n;
    const uint32_t sched = o ? o->schedule : G2_SCHED_GIVEN;
    const uint32_t flags = o ? o->flags : 0u;
    if (sched > G2_SCHED_LEARNED) return G2_ERR_INVALID;
    if (sched == G2_SCHED_SCORES && !(o && o->scores)) return G2_ERR_INVALID;
    if (sched == G2_SCHED_LEARNED && !ctx->d_model) return G2_ERR_INVALID;
    // MCE balances inside roots by handing branches to idle warps, which split
    // tasks cannot do: there the static split is only taken when asked for
    const bool split = nsrc > 0 && (sched == G2_SCHED_HEURISTIC || sched == G2_SCHED_LEARNED) &&
                       ((flags & G2_FLAG_SPLIT) ||
                        (!mce && sched == G2_SCHED_LEARNED && !(flags & G2_FLAG_NO_SPLIT)));
    // sum_i ceil(c_i / t) <= n + total / t = n + g * warps
    const uint32_t gran = (o && o->split_granularity) ? std::min<uint32_t>(o->split_granularity, 1024u) : 4u;
    const uint64_t cap = split ? nsrc + (uint64_t)gran * nwarps + 64 : nsrc;
    uint64_t tc = ctx->tasks_cap;
    int rc = grow(ctx, ctx->d_tasks, tc, cap, "tasks");
    if (rc) return rc;
    if (tc != ctx->tasks_cap || !ctx->d_defer) {
        // three deferred-task lists with stride tasks_cap
        if (ctx->d_defer) cudaFree(ctx->d_defer);
        ctx->d_defer = nullptr;
        G2_TRY(cudaMalloc(&ctx->d_defer, sizeof(uint32_t) * 3 * std::max<uint64_t>(tc, 1)));
    }
    ctx->tasks_cap = tc;
    tl->cap = nsrc;
    tl->split = false;
    const bool reorder = sched != G2_SCHED_GIVEN && nsrc >= 2;
    uint32_t *roots = ctx->d_tasks;
    if (reorder) {
        rc = grow(ctx, ctx->d_roots, ctx->roots_cap, nsrc, "roots");
        if (rc) return rc;
        roots = ctx->d_roots;
    }
    if (!sources) {
        iota_kernel<<<ctx->sm_count * 4, 256, 0, st>>>(roots, nsrc);
        ctx->launches++;
    } else if (nsrc) {
        G2_TRY(cudaMemcpyAsync(roots, sources, sizeof(uint32_t) * nsrc,
                               on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st));
    }
    if (!reorder) return G2_OK;
    rc = grow(ctx, ctx->d_keys, ctx->keys_cap, cap, "keys");
    if (!rc) rc = grow(ctx, ctx->d_keys2, ctx->keys2_cap, cap, "keys2");
    if (!rc) rc = grow(ctx, ctx->d_cost, ctx->cost_cap, nsrc, "cost");
    if (!rc && !ctx->d_total) rc = grow(ctx, ctx->d_total, ctx->total_cap, 2, "total");
    if (rc) return rc;
    // ---- cost per root
    G2_TRY(cudaMemsetAsync(ctx->d_total, 0, sizeof(float), st));
    if (sched == G2_SCHED_HEURISTIC) {
        heuristic_cost_kernel<<<ctx->sm_count * 4, 256, 0, st>>>(ctx->d_rp, ctx->d_fo, roots, nsrc, ctx->d_cost,
                                                                ctx->d_total);
        ctx->launches++;
    } else if (sched == G2_SCHED_LEARNED) {
        // features depend on the graph only: computed once per loaded graph (and
        // core numbers), then every run is MLP inference over the task list
        if (!ctx->feat_valid) {
            rc = grow(ctx, ctx->d_feat, ctx->feat_cap, (uint64_t)G2_MODEL_FEATURES * std::max<uint64_t>(ctx->n, 1),
                      "features");
            if (rc) return rc;
            cudaError_t e = g2::features_launch(ctx->d_rp, ctx->d_ci, ctx->d_fo, core_of(ctx), nullptr, ctx->n,
                                                ctx->d_feat, ctx->sm_count, st);
            if (e != cudaSuccess) return fail_cuda(ctx, e, "features_launch");
            ctx->launches++;
            ctx->feat_valid = true;
        }
        cudaError_t e = g2::score_launch(ctx->d_rp, ctx->d_ci, ctx->d_fo, core_of(ctx), roots, nsrc, ctx->d_feat,
                                         ctx->d_model, ctx->d_model + G2_MODEL_PARAMS, nullptr, ctx->d_cost,
                                         ctx->d_total, ctx->sm_count, st);
        if (e != cudaSuccess) return fail_cuda(ctx, e, "score_launch");
        ctx->launches++;
    } else {
        G2_TRY(cudaMemcpyAsync(ctx->d_cost, o->scores, sizeof(float) * nsrc, cudaMemcpyHostToDevice, st));
    }
    if (!split) {
        // one task per root, descending cost
        cost_keys_kernel<<<ctx->sm_count * 4, 256, 0, st>>>(ctx->d_cost, nsrc, ctx->d_keys);
        ctx->launches++;
        rc = sort_keys(ctx, nsrc, st);
        if (rc) return rc;
        gather_tasks_kernel<<<ctx->sm_count * 4, 256, 0, st>>>(ctx->d_keys2, roots, nullptr, nsrc, ctx->d_tasks,
                                                              nullptr);
        ctx->launches++;
        return G2_OK;
    }
    // ---- split heavy roots: tasks per root, offsets, expansion, sort, gather
    rc = grow(ctx, ctx->d_S, ctx->S_cap, 2 * nsrc, "split counts");
    if (!rc) rc = grow(ctx, ctx->d_part, ctx->part_cap, ctx->tasks_cap, "task parts");
    if (!rc) rc = grow(ctx, ctx->d_xroots, ctx->xroots_cap, cap, "expanded roots");
    if (!rc) rc = grow(ctx, ctx->d_xparts, ctx->xparts_cap, cap, "expanded parts");
    if (!rc && !ctx->d_ntask) rc = grow(ctx, ctx->d_ntask, ctx->ntask_cap, 1, "task count");
    if (rc) return rc;
    uint32_t *S = ctx->d_S, *off = ctx->d_S + nsrc;
    split_count_kernel<<<ctx->sm_count * 4, 256, 0, st>>>(ctx->d_cost, ctx->d_total, nsrc,
                                                         1.f / ((float)gran * (float)nwarps), S);
    size_t need = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need, S, off, (int)nsrc, st);
    rc = cub_space(ctx, need);
    if (rc) return rc;
    G2_TRY(cub::DeviceScan::ExclusiveSum(ctx->d_cub, need, S, off, (int)nsrc, st));
    G2_TRY(cudaMemsetAsync(ctx->d_keys, 0xff, sizeof(uint64_t) * cap, st));
    split_scatter_kernel<<<ctx->sm_count * 4, 256, 0, st>>>(roots, ctx->d_cost, S, off, nsrc, cap, ctx->d_xroots,
                                                           ctx->d_xparts, ctx->d_keys);
    split_total_kernel<<<1, 32, 0, st>>>(S, off, nsrc, cap, ctx->d_ntask);
    ctx->launches += 4;
    rc = sort_keys(ctx, cap, st);
    if (rc) return rc;
    gather_tasks_kernel<<<ctx->sm_count * 4, 256, 0, st>>>(ctx->d_keys2, ctx->d_xroots, ctx->d_xparts, cap,
                                                          ctx->d_tasks, ctx->d_part);
    ctx->launches++;
    tl->cap = cap;
    tl->split = true;
    return G2_OK;
}

}  // namespace g2rt

namespace {

int ensure_scratch(g2_ctx *ctx) {
    if (ctx->d_scratch) return G2_OK;
    uint64_t words = ctx->scratch_bytes / 4;
    words &= ~63ull;
    G2_TRY(cudaMalloc(&ctx->d_scratch, words * 4));
    ctx->scratch_words = words;
    return G2_OK;
}

// Device counters: queue heads of the passes, deferred-list sizes, hand-off
// record / pool allocation and the record queue.
constexpr int kCtrHead = 0;    // 3 queue heads
constexpr int kCtrDefer = 16;  // 3 deferred-list sizes
constexpr int kCtrRec = 19;    // records reserved
constexpr int kCtrPool = 20;   // pool units (64 words) used
constexpr int kCtrSpillDefer = 21;  // entries the host-spill pass could not hold
constexpr int kCtrQueue = 24;  // record queue: claimed, busy warps, idle warps
constexpr int kCtrWords = 40;

// MCE hand-off buffers and defaults.
constexpr uint64_t kRecordBytes = 1ull << 30;   // records (8 M plan-walk records, 16 M+ MCE records)
constexpr uint64_t kPoolBytes = 64ull << 20;    // rows of roots whose tasks handed off work
constexpr uint64_t kMaxRecords = kRecordBytes / 32;  // slots at the smallest stride (8 words)
constexpr uint32_t kSpillKcycles = 20;          // default check interval (x1000 SM cycles)
constexpr uint64_t kWaitCycles = 1ull << 37;    // longest wait for a record (~70 s of SM clock)

int ensure_handoff(g2_ctx *ctx, cudaStream_t st) {
    if (ctx->d_rec) return G2_OK;
    G2_TRY(cudaMalloc(&ctx->d_rec, kRecordBytes));
    G2_TRY(cudaMalloc(&ctx->d_pool, kPoolBytes));
    G2_TRY(cudaMalloc(&ctx->d_ready, sizeof(uint32_t) * kMaxRecords));
    G2_TRY(cudaMalloc(&ctx->d_epoch, sizeof(uint32_t)));
    // a ready word must never match a run's epoch by accident (a waiting warp
    // polls the ready word of a slot before it is reserved): ready words start
    // at 0, and every run bumps the device epoch, which skips 0, in stream order
    G2_TRY(cudaMemsetAsync(ctx->d_ready, 0, sizeof(uint32_t) * kMaxRecords, st));
    G2_TRY(cudaMemsetAsync(ctx->d_epoch, 0, sizeof(uint32_t), st));
    return G2_OK;
}

int ensure_counters(g2_ctx *ctx) {
    if (!ctx->d_ctr) G2_TRY(cudaMalloc(&ctx->d_ctr, sizeof(unsigned long long) * kCtrWords));
    if (!ctx->d_status) G2_TRY(cudaMalloc(&ctx->d_status, sizeof(int)));
    if (!ctx->d_deadline) G2_TRY(cudaMalloc(&ctx->d_deadline, sizeof(unsigned long long)));
    return G2_OK;
}

}  // namespace

namespace g2rt {

int status_to_code(int st) {
    if (st & g2::kStatusDeferOverflow) return G2_ERR_OVERFLOW;
    if (st & g2::kStatusStackOverflow) return G2_ERR_OVERFLOW;
    if (st & g2::kStatusBadPlan) return G2_ERR_INVALID;
    if (st & g2::kStatusHistOverflow) return G2_ERR_HIST;
    if (st & g2::kStatusWaitLimit) return G2_ERR_TIMEOUT;
    if (st & g2::kStatusDeadline) return G2_ERR_DEADLINE;
    return G2_OK;
}

}  // namespace g2rt

namespace {

// Events for pass timing and the device work counter, as the flags ask.
int prepare_flags(g2_ctx *ctx, uint32_t flags, cudaStream_t st) {
    ctx->timed = (flags & G2_FLAG_TIME_KERNELS) != 0;
    ctx->timed_passes = 0;
    ctx->last_stream = st;
    if (ctx->timed && !ctx->ev[0]) {
        for (auto &e : ctx->ev) G2_TRY(cudaEventCreate(&e));
    }
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

// Per-task outputs of the last run: zeroed device buffers of tasks_cap entries.
int prepare_root_outputs(g2_ctx *ctx, bool nodes, bool cost, cudaStream_t st) {
    if (nodes) {
        int rc = grow(ctx, ctx->d_root_nodes, ctx->root_nodes_cap, ctx->tasks_cap, "root nodes");
        if (rc) return rc;
        G2_TRY(cudaMemsetAsync(ctx->d_root_nodes, 0, sizeof(uint64_t) * ctx->tasks_cap, st));
    }
    if (cost) {
        int rc = grow(ctx, ctx->d_root_cost, ctx->root_cost_cap, ctx->tasks_cap, "root cost");
        if (rc) return rc;
        G2_TRY(cudaMemsetAsync(ctx->d_root_cost, 0, sizeof(uint64_t) * ctx->tasks_cap, st));
    }
    return G2_OK;
}

// Sum per-task outputs into per-source arrays (caller's order).  Synchronous.
int gather_root_outputs(g2_ctx *ctx, const uint32_t *sources, uint64_t nsrc, uint64_t *nodes_out,
                        uint64_t *cost_out) {
    if (!nodes_out && !cost_out) return G2_OK;
    const uint64_t cap = ctx->last_cap;
    std::vector<uint32_t> tasks(cap);
    std::vector<uint64_t> v(cap);
    G2_TRY(cudaMemcpy(tasks.data(), ctx->d_tasks, sizeof(uint32_t) * cap, cudaMemcpyDeviceToHost));
    uint64_t used = cap;
    if (ctx->last_split) {
        unsigned long long t = 0;
        G2_TRY(cudaMemcpy(&t, ctx->d_ntask, sizeof(t), cudaMemcpyDeviceToHost));
        used = t;
    }
    std::unordered_map<uint32_t, uint64_t> pos;
    if (sources)
        for (uint64_t i = nsrc; i-- > 0;) pos[sources[i]] = i;  // first occurrence wins
    auto index_of = [&](uint32_t root) -> uint64_t {
        if (!sources) return root;
        auto it = pos.find(root);
        return it == pos.end() ? ~0ull : it->second;
    };
    for (int which = 0; which < 2; which++) {
        uint64_t *out = which == 0 ? nodes_out : cost_out;
        uint64_t *dev = which == 0 ? ctx->d_root_nodes : ctx->d_root_cost;
        if (!out) continue;
        G2_TRY(cudaMemcpy(v.data(), dev, sizeof(uint64_t) * cap, cudaMemcpyDeviceToHost));
        memset(out, 0, sizeof(uint64_t) * nsrc);
        for (uint64_t i = 0; i < used; i++) {
            const uint64_t j = index_of(tasks[i]);
            if (j < nsrc) out[j] += v[i];
        }
    }
    return G2_OK;
}

// Optional L2 persistence window over the tail of the column array (the dense
// core's adjacency: ids are in degeneracy order) for the launches enqueued
// while it is set on the caller's stream.  The persisting-L2 limit it sets is a
// resource limit of this process's CUDA context and ends with it.
struct L2Window {
    cudaStream_t st = nullptr;
    bool on = false;
    L2Window(g2_ctx *ctx, cudaStream_t s, uint32_t flags) : st(s) {
        if (!(flags & G2_FLAG_L2_PERSIST) || !s || !ctx->m) return;
        int max_win = 0, max_persist = 0;
        if (cudaDeviceGetAttribute(&max_win, cudaDevAttrMaxAccessPolicyWindowSize, ctx->device) != cudaSuccess ||
            cudaDeviceGetAttribute(&max_persist, cudaDevAttrMaxPersistingL2CacheSize, ctx->device) != cudaSuccess ||
            max_win <= 0 || max_persist <= 0) {
            cudaGetLastError();
            return;
        }
        if (cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, (size_t)max_persist) != cudaSuccess) {
            cudaGetLastError();
            return;
        }
        const uint64_t bytes = std::min<uint64_t>(ctx->m * 4ull, (uint64_t)max_win);
        cudaStreamAttrValue v{};
        v.accessPolicyWindow.base_ptr = reinterpret_cast<char *>(ctx->d_ci) + (ctx->m * 4ull - bytes);
        v.accessPolicyWindow.num_bytes = bytes;
        v.accessPolicyWindow.hitRatio = std::min(1.0f, (float)max_persist / (float)bytes);
        v.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
        v.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
        on = cudaStreamSetAttribute(st, cudaStreamAttributeAccessPolicyWindow, &v) == cudaSuccess;
        if (!on) cudaGetLastError();
    }
    ~L2Window() {
        if (!on) return;
        cudaStreamAttrValue v{};
        v.accessPolicyWindow.num_bytes = 0;
        cudaStreamSetAttribute(st, cudaStreamAttributeAccessPolicyWindow, &v);
    }
};

// Enqueue the MCE passes; counters land in d_out.
}  // namespace

namespace g2rt {

int mce_enqueue(g2_ctx *ctx, const TaskList &tl, const g2_opts *o, unsigned long long *d_out, uint32_t hist_len,
                uint64_t *d_root_nodes, uint64_t *d_root_cost, cudaStream_t st, uint64_t *d_root_cliques) {
    int rc = ensure_scratch(ctx);
    if (rc) return rc;
    rc = ensure_counters(ctx);
    if (rc) return rc;
    if (ctx->max_fwd > 32u * 32u * 8u) return G2_ERR_UNSUPPORTED;
    const uint32_t flags = o ? o->flags : 0u;
    const uint32_t deadline_ms = o ? o->deadline_ms : 0u;
    // a run with a time budget drops unfinished roots whole, which needs every
    // root walked by one warp: no hand-off
    const bool spill = !(flags & G2_FLAG_NO_SPILL) && !deadline_ms;
    if (spill) {
        rc = ensure_handoff(ctx, st);
        if (rc) return rc;
    }
    G2_TRY(cudaMemsetAsync(ctx->d_ctr, 0, sizeof(unsigned long long) * kCtrWords, st));
    G2_TRY(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), st));
    G2_TRY(cudaMemsetAsync(d_out, 0, sizeof(unsigned long long) * (1 + hist_len), st));
    rc = prepare_flags(ctx, flags, st);
    if (rc) return rc;
    const int wpb = default_warps(o);
    const int blocks = default_blocks(ctx, o, wpb, g2::mce_blocks_per_sm(1, wpb, (flags & G2_FLAG_WORK_MODEL) != 0));
    // records hold rows of the WPL=1 main pass: at most 32 words
    const uint32_t rec_words = std::min<uint32_t>((ctx->max_fwd + 31u) / 32u, 32u);
    const uint32_t rec_stride = (4u + 3u * std::max<uint32_t>(rec_words, 1u) + 3u) & ~3u;
    const uint64_t spill_cycles =
        spill ? 1000ull * ((o && o->spill_kcycles) ? o->spill_kcycles : kSpillKcycles) : 0ull;
    if (spill) {
        cudaError_t e = g2::epoch_bump(ctx->d_epoch, st);
        if (e != cudaSuccess) return fail_cuda(ctx, e, "epoch_bump");
        ctx->launches++;
    }
    g2::MceArgs base{};
    base.rp = ctx->d_rp;
    base.ci = ctx->d_ci;
    base.fo = ctx->d_fo;
    base.tasks = ctx->d_tasks;
    base.task_part = tl.split ? ctx->d_part : nullptr;
    base.split_depth = (o && o->split_depth) ? o->split_depth : 2u;
    base.root_cost = d_root_cost;
    base.hist_len = hist_len;
    base.scratch = ctx->d_scratch;
    base.out = d_out;
    base.deferred_cap = ctx->tasks_cap;
    base.root_nodes = d_root_nodes;
    base.root_cliques = d_root_cliques;
    base.status = ctx->d_status;
    base.work = (flags & G2_FLAG_WORK_MODEL) ? ctx->d_work : nullptr;
    base.records = ctx->d_rec;
    base.ready = ctx->d_ready;
    base.nrec = ctx->d_ctr + kCtrRec;
    base.rec_cap = spill ? std::min<uint64_t>(kRecordBytes / (4ull * rec_stride), g2::kRecordBit - 1u) : 0;
    base.rec_stride = rec_stride;
    base.rec_words = rec_words;
    base.pool = ctx->d_pool;
    base.npool = ctx->d_ctr + kCtrPool;
    base.pool_cap = spill ? kPoolBytes / 4 : 0;
    base.qctl = ctx->d_ctr + kCtrQueue;
    base.epoch_dev = spill ? ctx->d_epoch : nullptr;
    base.wait_cycles = (o && o->wait_cycles) ? o->wait_cycles : kWaitCycles;
    if (deadline_ms) {
        cudaError_t e = g2::deadline_set(ctx->d_deadline, 1000000ull * deadline_ms, st);
        if (e != cudaSuccess) return fail_cuda(ctx, e, "deadline_set");
        ctx->launches++;
        base.deadline = ctx->d_deadline;
    }
    if (ctx->timed) G2_TRY(cudaEventRecord(ctx->ev[0], st));
    L2Window l2(ctx, st, flags);
    {  // main pass: every task, WPL=1, one slab per resident warp; long walks
       // hand branches to idle warps through the record queue
        g2::MceArgs a = base;
        a.head = ctx->d_ctr + kCtrHead;
        a.chunk = (o && o->chunk) ? o->chunk : 1u;
        a.words_per_warp = (ctx->scratch_words / ((uint64_t)blocks * wpb)) & ~63ull;
        a.deferred = ctx->d_defer;
        a.ndeferred = ctx->d_ctr + kCtrDefer;
        a.spill_cycles = spill_cycles;
        a.ntasks = tl.cap;
        a.ntasks_dev = tl.split ? ctx->d_ntask : nullptr;
        cudaError_t e = g2::mce_launch(1, a, blocks, wpb, st);
        if (e != cudaSuccess) return fail_cuda(ctx, e, "mce_launch");
        ctx->launches++;
    }
    if (ctx->timed) G2_TRY(cudaEventRecord(ctx->ev[1], st));
    // deferred entries: 2 warps per SM with WPL for the widest root, then one
    // warp owning the whole slab; neither spills
    struct Pass {
        int blocks, wpb, wpl;
    } passes[2] = {{ctx->sm_count, 2, wpl_for(ctx->max_fwd)}, {1, 1, wpl_for(ctx->max_fwd)}};
    for (int k = 0; k < 2; k++) {
        g2::MceArgs a = base;
        a.task_index = ctx->d_defer + (uint64_t)k * ctx->tasks_cap;
        a.ntasks_dev = ctx->d_ctr + kCtrDefer + k;
        a.head = ctx->d_ctr + kCtrHead + 1 + k;
        a.chunk = 1;
        a.words_per_warp = (ctx->scratch_words / ((uint64_t)passes[k].blocks * passes[k].wpb)) & ~63ull;
        a.deferred = ctx->d_defer + (uint64_t)(k + 1) * ctx->tasks_cap;
        a.ndeferred = ctx->d_ctr + kCtrDefer + k + 1;
        cudaError_t e = g2::mce_launch(passes[k].wpl, a, passes[k].blocks, passes[k].wpb, st);
        if (e != cudaSuccess) return fail_cuda(ctx, e, "mce_launch");
        if (ctx->timed) G2_TRY(cudaEventRecord(ctx->ev[k + 2], st));
        ctx->launches++;
    }
    ctx->last_mce = base;
    ctx->last_mce_wpl = wpl_for(ctx->max_fwd);
    if (ctx->timed) ctx->timed_passes = 3;
    return G2_OK;
}

}  // namespace g2rt

namespace {

// After a synchronous MCE run: entries that no device slab held (deferred by the
// single-warp pass) run once more with one warp whose slab is managed memory of
// g2_set_host_spill's size (allocated on first need; its pages move to the GPU
// as they are touched and back to the host if device memory runs out), adding
// to the same outputs.  Returns G2_ERR_OVERFLOW if entries remain.  Managed
// rather than mapped pinned memory: the walk's many small reads stay in device
// memory while the slab is in use.
}  // namespace

namespace g2rt {

// The spill slab (managed memory of g2_set_host_spill's size), allocated or
// resized on first need.
static int ensure_spill_slab(g2_ctx *ctx) {
    if (ctx->h_spill_bytes == ctx->host_spill_bytes) return G2_OK;
    if (ctx->h_spill) cudaFree(ctx->h_spill);
    ctx->h_spill = nullptr;
    ctx->h_spill_bytes = 0;
    G2_TRY(cudaMallocManaged(&ctx->h_spill, ctx->host_spill_bytes));
    ctx->h_spill_bytes = ctx->host_spill_bytes;
    return G2_OK;
}

// The spill pass over the one-warp pass's leftover entries (count read on the
// device: the kernel exits at once when there are none); its own leftovers
// go to kCtrSpillDefer.
static int launch_spill_pass(g2_ctx *ctx, cudaStream_t st) {
    g2::MceArgs a = ctx->last_mce;
    a.scratch = static_cast<uint32_t *>(ctx->h_spill);
    // the root's clique-size counters go to the idle device scratch
    a.hist_dev = reinterpret_cast<unsigned long long *>(ctx->d_scratch);
    a.words_per_warp = (ctx->h_spill_bytes / 4) & ~63ull;
    a.task_index = ctx->d_defer + 2 * ctx->tasks_cap;
    a.ntasks_dev = ctx->d_ctr + kCtrDefer + 2;
    a.head = ctx->d_ctr + kCtrHead + 3;
    a.chunk = 1;
    a.deferred = ctx->d_defer;  // list 0 is free again
    a.ndeferred = ctx->d_ctr + kCtrSpillDefer;
    a.spill_cycles = 0;
    G2_TRY(cudaMemsetAsync(a.head, 0, sizeof(unsigned long long), st));
    G2_TRY(cudaMemsetAsync(a.ndeferred, 0, sizeof(unsigned long long), st));
    cudaError_t e = g2::mce_launch(ctx->last_mce_wpl, a, 1, 1, st);
    if (e != cudaSuccess) return fail_cuda(ctx, e, "mce_launch (host spill)");
    ctx->launches++;
    return G2_OK;
}

int mce_host_spill(g2_ctx *ctx, cudaStream_t st) {
    unsigned long long left = 0;
    G2_TRY(cudaMemcpy(&left, ctx->d_ctr + kCtrDefer + 2, sizeof(left), cudaMemcpyDeviceToHost));
    if (!left) return G2_OK;
    if (!ctx->host_spill_bytes || left > ctx->tasks_cap) return G2_ERR_OVERFLOW;
    if (ctx->scratch_words < 2ull * (ctx->max_fwd + 2)) return G2_ERR_OVERFLOW;  // room for the histogram
    int rc = ensure_spill_slab(ctx);
    if (!rc) rc = launch_spill_pass(ctx, st);
    if (rc) return rc;
    G2_TRY(cudaMemcpy(&left, ctx->d_ctr + kCtrSpillDefer, sizeof(left), cudaMemcpyDeviceToHost));
    return left ? G2_ERR_OVERFLOW : G2_OK;
}

// Device-stream MCE runs: the same spill pass in stream order, without a host
// read of the leftover count, then a one-thread kernel that flags entries still
// left (read with g2_run_status).  The slab must exist before a CUDA graph
// capture: inside one, a slab not yet allocated means no spill pass.
int mce_stream_spill(g2_ctx *ctx, cudaStream_t st) {
    const unsigned long long *left = ctx->d_ctr + kCtrDefer + 2;
    bool can = ctx->host_spill_bytes && ctx->scratch_words >= 2ull * (ctx->max_fwd + 2);
    if (can && ctx->h_spill_bytes != ctx->host_spill_bytes) {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        G2_TRY(cudaStreamIsCapturing(st, &cs));
        if (cs != cudaStreamCaptureStatusNone) can = false;
        else if (int rc = ensure_spill_slab(ctx)) return rc;
    }
    if (can) {
        int rc = launch_spill_pass(ctx, st);
        if (rc) return rc;
        left = ctx->d_ctr + kCtrSpillDefer;
    }
    cudaError_t e = g2::flag_left(left, ctx->d_status, st);
    if (e != cudaSuccess) return fail_cuda(ctx, e, "flag_left");
    ctx->launches++;
    return G2_OK;
}

}  // namespace g2rt

namespace {

// Persistent-grid geometry of the match kernel.
void match_geometry(g2_ctx *ctx, const g2_opts *o, int *wpl, int *wpb, int *blocks, uint32_t *p0_words) {
    *wpl = wpl_for(ctx->max_fwd);
    *wpb = default_warps(o);
    const bool metrics = o && (o->flags & G2_FLAG_WORK_MODEL);
    const bool clique = ctx->clique_plan && !(o && o->intersect_mode == 1);
    *p0_words = g2::match_p0_words(*wpl, clique, ctx->plan.k, metrics);
    while (*wpb > 1 && g2::match_smem_bytes(*wpl, *wpb, *p0_words) > 200 * 1024) *wpb /= 2;
    *blocks = default_blocks(
        ctx, o, *wpb, g2::match_blocks_per_sm(*wpl, *wpb, metrics, o ? (int)o->ctas_per_sm : 0, *p0_words));
}

}  // namespace

namespace g2rt {

int match_enqueue(g2_ctx *ctx, const TaskList &tl, const g2_opts *o, unsigned long long *d_out,
                  uint64_t *d_root_nodes, uint64_t *d_root_cost, cudaStream_t st) {
    int rc = ensure_scratch(ctx);
    if (rc) return rc;
    rc = ensure_counters(ctx);
    if (rc) return rc;
    G2_TRY(cudaMemsetAsync(ctx->d_ctr, 0, sizeof(unsigned long long) * kCtrWords, st));
    G2_TRY(cudaMemsetAsync(ctx->d_status, 0, sizeof(int), st));
    G2_TRY(cudaMemsetAsync(d_out, 0, sizeof(unsigned long long), st));
    const uint32_t flags = o ? o->flags : 0u;
    rc = prepare_flags(ctx, flags, st);
    if (rc) return rc;
    int wpl, wpb, blocks;
    uint32_t p0_words;
    match_geometry(ctx, o, &wpl, &wpb, &blocks, &p0_words);
    g2::MatchArgs a{};
    a.p0_words = p0_words;
    a.rp = ctx->d_rp;
    a.ci = ctx->d_ci;
    a.fo = ctx->d_fo;
    a.tasks = ctx->d_tasks;
    a.task_part = tl.split ? ctx->d_part : nullptr;
    a.root_cost = d_root_cost;
    a.ntasks = tl.cap;
    a.ntasks_dev = tl.split ? ctx->d_ntask : nullptr;
    a.head = ctx->d_ctr;
    a.chunk = (o && o->chunk) ? o->chunk : 4u;
    a.scratch = ctx->d_scratch;
    a.words_per_warp = (ctx->scratch_words / ((uint64_t)blocks * wpb)) & ~63ull;
    if (a.words_per_warp / (ctx->plan.k > 2 ? ctx->plan.k - 2 : 1) < 64) return G2_ERR_OVERFLOW;
    a.out = d_out;
    a.root_nodes = d_root_nodes;
    a.status = ctx->d_status;
    a.work = (flags & G2_FLAG_WORK_MODEL) ? ctx->d_work : nullptr;
    const bool clique = ctx->clique_plan && !(o && o->intersect_mode == 1);
    const uint32_t deadline_ms = o ? o->deadline_ms : 0u;
    if (deadline_ms) {  // time budget: unfinished roots are dropped whole, so no hand-off
        cudaError_t ed = g2::deadline_set(ctx->d_deadline, 1000000ull * deadline_ms, st);
        if (ed != cudaSuccess) return fail_cuda(ctx, ed, "deadline_set");
        ctx->launches++;
        a.deadline = ctx->d_deadline;
    }
    // plan walks (non-clique plans) hand pending work to idle warps
    if (!clique && !(flags & G2_FLAG_NO_SPILL) && !deadline_ms) {
        rc = ensure_handoff(ctx, st);
        if (rc) return rc;
        cudaError_t eb = g2::epoch_bump(ctx->d_epoch, st);
        if (eb != cudaSuccess) return fail_cuda(ctx, eb, "epoch_bump");
        ctx->launches++;
        a.records = ctx->d_rec;
        a.ready = ctx->d_ready;
        a.nrec = ctx->d_ctr + kCtrRec;
        a.rec_stride = g2::kMatchRecordWords;
        a.rec_cap = std::min<uint64_t>(kRecordBytes / (4ull * a.rec_stride), g2::kRecordBit - 1u);
        a.qctl = ctx->d_ctr + kCtrQueue;
        a.epoch_dev = ctx->d_epoch;
        a.wait_cycles = (o && o->wait_cycles) ? o->wait_cycles : kWaitCycles;
        a.spill_cycles = 1000ull * ((o && o->spill_kcycles) ? o->spill_kcycles : kSpillKcycles);
    }
    if (ctx->timed) G2_TRY(cudaEventRecord(ctx->ev[0], st));
    L2Window l2(ctx, st, flags);
    cudaError_t e = g2::match_launch(ctx->plan, a, blocks, wpb, st, clique, wpl, o ? (int)o->ctas_per_sm : 0);
    if (e != cudaSuccess) return fail_cuda(ctx, e, "match_launch");
    if (ctx->timed) G2_TRY(cudaEventRecord(ctx->ev[1], st));
    ctx->launches++;
    if (ctx->timed) ctx->timed_passes = 1;
    return G2_OK;
}

}  // namespace g2rt

namespace {

}  // namespace

namespace g2rt {

uint64_t mce_warps(g2_ctx *ctx, const g2_opts *o) {
    const int wpb = default_warps(o);
    const bool metrics = o && (o->flags & G2_FLAG_WORK_MODEL);
    return (uint64_t)default_blocks(ctx, o, wpb, g2::mce_blocks_per_sm(1, wpb, metrics)) * wpb;
}

}  // namespace g2rt

namespace {

}  // namespace

namespace g2rt {

uint64_t match_warps(g2_ctx *ctx, const g2_opts *o) {
    int wpl, wpb, blocks;
    uint32_t p0_words;
    match_geometry(ctx, o, &wpl, &wpb, &blocks, &p0_words);
    return (uint64_t)blocks * wpb;
}

}  // namespace g2rt

namespace {

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
        case G2_ERR_DEADLINE: return "time budget ran out (outputs hold the roots that finished)";
        default: return "unknown error";
    }
}

const char *g2_last_cuda_error(const g2_ctx *ctx) { return ctx ? ctx->cuda_err.c_str() : ""; }

uint64_t g2_last_launch_count(const g2_ctx *ctx) { return ctx ? ctx->launches : 0; }

int g2_pass_time_ms(g2_ctx *ctx, int pass, float *ms) {
    if (!ctx || !ms || pass < 0 || pass >= ctx->timed_passes || !ctx->timed) return G2_ERR_INVALID;
    G2_TRY(cudaEventSynchronize(ctx->ev[pass + 1]));
    G2_TRY(cudaEventElapsedTime(ms, ctx->ev[pass], ctx->ev[pass + 1]));
    return G2_OK;
}

int g2_reserve(g2_ctx *ctx, uint64_t max_sources) {
    if (!ctx) return G2_ERR_INVALID;
    G2_TRY(cudaSetDevice(ctx->device));
    if (!max_sources) max_sources = ctx->n;
    int rc = ensure_scratch(ctx);
    if (!rc) rc = ensure_counters(ctx);
    if (!rc) rc = ensure_handoff(ctx, nullptr);
    if (rc) return rc;
    if (max_sources) {
        // tasks of a run with heavy-root splits at the default granularity (4)
        // over the largest resident grid, the three deferred lists, the
        // schedule's keys, costs and root lists, and the sort's scratch
        const uint64_t cap = max_sources + 4ull * (uint64_t)ctx->sm_count * 64ull + 64ull;
        uint64_t tc = ctx->tasks_cap;
        rc = grow(ctx, ctx->d_tasks, tc, cap, "tasks");
        if (rc) return rc;
        if (tc != ctx->tasks_cap || !ctx->d_defer) {
            if (ctx->d_defer) cudaFree(ctx->d_defer);
            ctx->d_defer = nullptr;
            G2_TRY(cudaMalloc(&ctx->d_defer, sizeof(uint32_t) * 3 * std::max<uint64_t>(tc, 1)));
        }
        ctx->tasks_cap = tc;
        rc = grow(ctx, ctx->d_roots, ctx->roots_cap, max_sources, "roots");
        if (!rc) rc = grow(ctx, ctx->d_keys, ctx->keys_cap, cap, "keys");
        if (!rc) rc = grow(ctx, ctx->d_keys2, ctx->keys2_cap, cap, "keys2");
        if (!rc) rc = grow(ctx, ctx->d_cost, ctx->cost_cap, max_sources, "cost");
        if (!rc && !ctx->d_total) rc = grow(ctx, ctx->d_total, ctx->total_cap, 2, "total");
        if (!rc) rc = grow(ctx, ctx->d_S, ctx->S_cap, 2 * max_sources, "split counts");
        if (!rc) rc = grow(ctx, ctx->d_part, ctx->part_cap, ctx->tasks_cap, "task parts");
        if (!rc) rc = grow(ctx, ctx->d_xroots, ctx->xroots_cap, cap, "expanded roots");
        if (!rc) rc = grow(ctx, ctx->d_xparts, ctx->xparts_cap, cap, "expanded parts");
        if (!rc && !ctx->d_ntask) rc = grow(ctx, ctx->d_ntask, ctx->ntask_cap, 1, "task count");
        if (rc) return rc;
        size_t sort_need = 0, scan_need = 0;
        cub::DeviceRadixSort::SortKeys(nullptr, sort_need, ctx->d_keys, ctx->d_keys2, (int)cap, 0, 64);
        cub::DeviceScan::ExclusiveSum(nullptr, scan_need, ctx->d_S, ctx->d_S, (int)max_sources);
        rc = cub_space(ctx, std::max(sort_need, scan_need));
        if (rc) return rc;
    }
    G2_TRY(cudaDeviceSynchronize());
    return G2_OK;
}

int g2_degeneracy_order_device(g2_ctx *ctx, uint32_t *perm, uint32_t *core) {
    if (!ctx || !perm) return G2_ERR_INVALID;
    if (!ctx->d_rp) return G2_ERR_NO_GRAPH;
    G2_TRY(cudaSetDevice(ctx->device));
    const uint64_t n = ctx->n;
    if (n == 0) return G2_OK;
    uint32_t *d_perm = nullptr, *d_core = nullptr;
    G2_TRY(cudaMalloc(&d_perm, n * 4));
    cudaError_t e = cudaMalloc(&d_core, n * 4);
    uint64_t rounds = 0;
    if (e == cudaSuccess) e = g2::degeneracy_order_device(ctx->d_rp, ctx->d_ci, n, d_perm, d_core, ctx->sm_count, &rounds);
    if (e == cudaSuccess) e = cudaMemcpy(perm, d_perm, n * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && core) e = cudaMemcpy(core, d_core, n * 4, cudaMemcpyDeviceToHost);
    cudaFree(d_perm);
    cudaFree(d_core);
    if (e != cudaSuccess) return fail_cuda(ctx, e, "degeneracy_order_device");
    ctx->launches = 2 * rounds + 4;
    return G2_OK;
}

static int after_load(g2_ctx *ctx);

int g2_degeneracy_recode_device(g2_ctx *ctx, uint32_t *perm, uint32_t *core) {
    if (!ctx) return G2_ERR_INVALID;
    if (!ctx->d_rp) return G2_ERR_NO_GRAPH;
    G2_TRY(cudaSetDevice(ctx->device));
    const uint64_t n = ctx->n, m = ctx->m;
    if (n == 0) return G2_OK;
    if (n + 1 > (uint64_t)INT_MAX) return G2_ERR_UNSUPPORTED;
    uint64_t max_chunk = 1ull << 30;  // entries per segmented-sort call (CUB counts items in int)
    if (const char *env = getenv("G2_RECODE_CHUNK")) max_chunk = std::max<uint64_t>(strtoull(env, nullptr, 10), 1);
    uint32_t *d_perm = nullptr, *d_core = nullptr;
    uint64_t *nrp = nullptr;
    uint32_t *nci = nullptr;
    uint64_t rounds = 0;
    cudaError_t e = cudaMalloc(&d_perm, n * 4);
    if (e == cudaSuccess) e = cudaMalloc(&d_core, n * 4);
    if (e == cudaSuccess)
        e = g2::degeneracy_order_device(ctx->d_rp, ctx->d_ci, n, d_perm, d_core, ctx->sm_count, &rounds);
    if (e == cudaSuccess) e = g2::recode_device(ctx->d_rp, ctx->d_ci, n, m, d_perm, max_chunk, ctx->sm_count, &nrp, &nci);
    if (e == cudaSuccess && perm) e = cudaMemcpy(perm, d_perm, n * 4, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && core) e = cudaMemcpy(core, d_core, n * 4, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        cudaFree(d_perm);
        cudaFree(d_core);
        cudaFree(nrp);
        cudaFree(nci);
        return e == cudaErrorNotSupported ? G2_ERR_UNSUPPORTED : fail_cuda(ctx, e, "degeneracy recode");
    }
    // the recoded CSR becomes the context's graph
    if (ctx->owns_csr) {
        cudaFree(ctx->d_rp);
        cudaFree(ctx->d_ci);
    }
    ctx->d_rp = nrp;
    ctx->d_ci = nci;
    ctx->owns_csr = true;
    ctx->rp_cap = n + 1;
    ctx->ci_cap = std::max<uint64_t>(m, 1);
    int rc = after_load(ctx);
    // core numbers under the new names, for the learned schedule's features
    if (!rc) rc = grow(ctx, ctx->d_core, ctx->core_cap, n, "core");
    if (!rc) {
        rename_kernel<<<ctx->sm_count * 4, 256>>>(d_core, d_perm, n, ctx->d_core);
        e = cudaDeviceSynchronize();
        if (e != cudaSuccess) rc = fail_cuda(ctx, e, "core rename");
    }
    cudaFree(d_perm);
    cudaFree(d_core);
    if (rc) return rc;
    ctx->core_loaded = true;
    ctx->launches = 2 * rounds + 12;
    return G2_OK;
}

int g2_copy_csr(g2_ctx *ctx, uint64_t *row_ptrs, uint32_t *cols) {
    if (!ctx || !row_ptrs || (!cols && ctx->m)) return G2_ERR_INVALID;
    if (!ctx->d_rp) return G2_ERR_NO_GRAPH;
    G2_TRY(cudaSetDevice(ctx->device));
    G2_TRY(cudaMemcpy(row_ptrs, ctx->d_rp, 8 * (ctx->n + 1), cudaMemcpyDeviceToHost));
    if (ctx->m) G2_TRY(cudaMemcpy(cols, ctx->d_ci, 4 * ctx->m, cudaMemcpyDeviceToHost));
    return G2_OK;
}

int g2_set_host_spill(g2_ctx *ctx, uint64_t bytes) {
    if (!ctx || (bytes && bytes < (1u << 20))) return G2_ERR_INVALID;
    ctx->host_spill_bytes = bytes;
    return G2_OK;
}

int g2_last_spill_stats(g2_ctx *ctx, uint64_t *records, uint64_t *pool_bytes) {
    if (!ctx || !records || !pool_bytes || !ctx->d_ctr) return G2_ERR_INVALID;
    unsigned long long h[2] = {0, 0};
    G2_TRY(cudaStreamSynchronize(ctx->last_stream));
    G2_TRY(cudaMemcpy(h, ctx->d_ctr + kCtrRec, sizeof(h), cudaMemcpyDeviceToHost));
    *records = h[0];
    *pool_bytes = h[1] * 64ull * 4ull;
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
    void *bufs[] = {ctx->d_fo,     ctx->d_core,    ctx->d_scratch, ctx->d_tasks,  ctx->d_defer,      ctx->d_root_nodes,
                    ctx->d_root_cost, ctx->d_ctr,  ctx->d_status,  ctx->d_out,    ctx->d_keys,       ctx->d_keys2,
                    ctx->d_roots,  ctx->d_S,       ctx->d_part,    ctx->d_xroots, ctx->d_xparts,     ctx->d_cost,
                    ctx->d_total,  ctx->d_ntask,   ctx->d_cub,     ctx->d_model,  ctx->d_work,
                    ctx->d_feat,   ctx->d_rec,     ctx->d_pool,    ctx->d_ready,  ctx->d_goff,    ctx->d_fwdmax,
                    ctx->d_epoch,  ctx->d_deadline,
                    ctx->d_root_cliques, ctx->d_gcount};
    for (void *b : bufs)
        if (b) cudaFree(b);
    for (auto &e : ctx->ev)
        if (e) cudaEventDestroy(e);
    if (ctx->h_spill) cudaFree(ctx->h_spill);
    for (auto &h : ctx->view_host)
        if (h.first) cudaFreeHost(h.first);
    for (void *b : ctx->view_dev)
        if (b) cudaFree(b);
    g2rt::view_builder_free(ctx->view_builder);
    delete ctx;
    return G2_OK;
}

static int after_load(g2_ctx *ctx) {
    int rc = grow(ctx, ctx->d_fo, ctx->fo_cap, std::max<uint64_t>(ctx->n, 1), "forward offsets");
    if (rc) return rc;
    ctx->batch_off.clear();  // a batch load sets it again afterwards
    ctx->feat_valid = false;
    ctx->core_loaded = false;  // core numbers belong to the previous graph (buffer kept)
    if (!ctx->d_fwdmax) G2_TRY(cudaMalloc(&ctx->d_fwdmax, sizeof(unsigned int)));
    unsigned int *d_max = ctx->d_fwdmax;
    G2_TRY(cudaMemset(d_max, 0, sizeof(unsigned int)));
    if (ctx->n) forward_offsets_kernel<<<ctx->sm_count * 4, 256>>>(ctx->d_rp, ctx->d_ci, ctx->n, ctx->d_fo, d_max);
    ctx->launches++;
    unsigned int h = 0;
    cudaError_t e = cudaMemcpy(&h, d_max, sizeof(unsigned int), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail_cuda(ctx, e, "fwd_max");
    ctx->max_fwd = h;
    return G2_OK;
}

int g2_load_csr(g2_ctx *ctx, const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n, uint64_t m) {
    if (!ctx || !row_ptrs || (!cols && m) || n >= (1ull << 32)) return G2_ERR_INVALID;
    if (row_ptrs[n] != m) return G2_ERR_INVALID;
    G2_TRY(cudaSetDevice(ctx->device));
    // owned CSR buffers are kept and reused while large enough (no free/alloc,
    // which synchronise the device, on a reload of a graph of the same size)
    if (!ctx->owns_csr) {
        ctx->d_rp = nullptr;
        ctx->d_ci = nullptr;
        ctx->rp_cap = ctx->ci_cap = 0;
    }
    ctx->owns_csr = true;
    if (ctx->rp_cap < n + 1) {
        if (ctx->d_rp) cudaFree(ctx->d_rp);
        ctx->d_rp = nullptr;
        ctx->rp_cap = 0;
        G2_TRY(cudaMalloc(&ctx->d_rp, sizeof(uint64_t) * (n + 1)));
        ctx->rp_cap = n + 1;
    }
    if (ctx->ci_cap < std::max<uint64_t>(m, 1)) {
        if (ctx->d_ci) cudaFree(ctx->d_ci);
        ctx->d_ci = nullptr;
        ctx->ci_cap = 0;
        G2_TRY(cudaMalloc(&ctx->d_ci, sizeof(uint32_t) * std::max<uint64_t>(m, 1)));
        ctx->ci_cap = std::max<uint64_t>(m, 1);
    }
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
        ctx->rp_cap = ctx->ci_cap = 0;
    }
    ctx->d_rp = const_cast<uint64_t *>(d_row_ptrs);
    ctx->d_ci = const_cast<uint32_t *>(d_cols);
    ctx->owns_csr = false;
    ctx->n = n;
    ctx->m = m;
    return after_load(ctx);
}

int g2_load_core(g2_ctx *ctx, const uint32_t *core) {
    if (!ctx || !core) return G2_ERR_INVALID;
    if (!ctx->d_rp) return G2_ERR_NO_GRAPH;
    G2_TRY(cudaSetDevice(ctx->device));
    int rc = grow(ctx, ctx->d_core, ctx->core_cap, std::max<uint64_t>(ctx->n, 1), "core");
    if (rc) return rc;
    ctx->feat_valid = false;
    if (ctx->n) G2_TRY(cudaMemcpy(ctx->d_core, core, sizeof(uint32_t) * ctx->n, cudaMemcpyHostToDevice));
    ctx->core_loaded = true;
    return G2_OK;
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
        if (i > 0 && (p->bn_count[i] == 0 || p->bn_count[i] > k)) return G2_ERR_INVALID;
        if (p->cond_count[u] > k) return G2_ERR_INVALID;
        d.bn_count[i] = p->bn_count[i];
        for (uint32_t j = 0; j < p->bn_count[i]; j++) {
            if (p->bn[i][j] >= k) return G2_ERR_INVALID;
            uint32_t pos = p->id2order[p->bn[i][j]];
            if (pos >= i) return G2_ERR_INVALID;
            d.bn_pos[i][j] = pos;
        }
        d.cond_count[i] = p->cond_count[u];
        uint32_t larger = 0;
        for (uint32_t j = 0; j < p->cond_count[u]; j++) {
            if (p->cond[u][j][1] >= k) return G2_ERR_INVALID;
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
    TaskList tl;
    int rc = prepare_tasks(ctx, d_sources, nsrc, true, opts, mce_warps(ctx, opts), st, &tl, true);
    if (rc) return rc;
    ctx->last_split = tl.split;
    ctx->last_cap = tl.cap;
    rc = mce_enqueue(ctx, tl, opts, reinterpret_cast<unsigned long long *>(d_out), hist_len, nullptr, nullptr, st);
    if (rc) return rc;
    return mce_stream_spill(ctx, st);
}

int g2_run_status(g2_ctx *ctx, void *stream) {
    if (!ctx) return G2_ERR_INVALID;
    if (!ctx->d_status) return G2_OK;  // nothing has run
    G2_TRY(cudaSetDevice(ctx->device));
    G2_TRY(cudaStreamSynchronize((cudaStream_t)stream));
    int status = 0;
    G2_TRY(cudaMemcpy(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    return status_to_code(status);
}

int g2_mce_run(g2_ctx *ctx, const uint32_t *sources, uint64_t nsrc, const g2_opts *opts, uint64_t *count,
               uint64_t *hist, uint32_t hist_len) {
    if (!ctx || !count || (hist && hist_len == 0)) return G2_ERR_INVALID;
    if (!ctx->d_rp) return G2_ERR_NO_GRAPH;
    G2_TRY(cudaSetDevice(ctx->device));
    ctx->launches = 0;
    const uint32_t hl = hist ? hist_len : 0u;  // no histogram requested: count only
    cudaStream_t st = nullptr;
    g2_opts o2{};
    if (opts) o2 = *opts;
    if (o2.work_bytes) o2.flags |= G2_FLAG_WORK_MODEL;
    TaskList tl;
    int rc = prepare_tasks(ctx, sources, nsrc, false, &o2, mce_warps(ctx, &o2), st, &tl, true);
    if (rc) return rc;
    if (!sources) nsrc = ctx->n;
    ctx->last_split = tl.split;
    ctx->last_cap = tl.cap;
    rc = prepare_root_outputs(ctx, o2.root_nodes != nullptr, o2.root_cost != nullptr, st);
    if (rc) return rc;
    rc = grow(ctx, ctx->d_out, ctx->out_cap, 1 + hl, "out");
    if (rc) return rc;
    rc = mce_enqueue(ctx, tl, &o2, ctx->d_out, hl, o2.root_nodes ? ctx->d_root_nodes : nullptr,
                     o2.root_cost ? ctx->d_root_cost : nullptr, st);
    if (rc) return rc;
    rc = mce_host_spill(ctx, st);  // adds to the outputs: read them after it
    if (rc) return rc;
    std::vector<unsigned long long> h(1 + hl);
    int status = 0;
    G2_TRY(cudaMemcpy(h.data(), ctx->d_out, sizeof(unsigned long long) * (1 + hl), cudaMemcpyDeviceToHost));
    G2_TRY(cudaMemcpy(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    *count = h[0];
    if (hist)
        for (uint32_t s = 0; s < hist_len; s++) hist[s] = h[1 + s];
    if (o2.work_bytes) {
        rc = g2_last_work_bytes(ctx, o2.work_bytes);
        if (rc) return rc;
    }
    rc = gather_root_outputs(ctx, sources, nsrc, o2.root_nodes, o2.root_cost);
    if (rc) return rc;
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
    TaskList tl;
    int rc = prepare_tasks(ctx, d_sources, nsrc, true, opts, match_warps(ctx, opts), st, &tl, false);
    if (rc) return rc;
    ctx->last_split = tl.split;
    ctx->last_cap = tl.cap;
    return match_enqueue(ctx, tl, opts, reinterpret_cast<unsigned long long *>(d_out), nullptr, nullptr, st);
}

int g2_match_run(g2_ctx *ctx, const uint32_t *sources, uint64_t nsrc, const g2_opts *opts, uint64_t *count) {
    if (!ctx || !count) return G2_ERR_INVALID;
    if (!ctx->d_rp) return G2_ERR_NO_GRAPH;
    if (!ctx->has_plan) return G2_ERR_NO_PLAN;
    G2_TRY(cudaSetDevice(ctx->device));
    ctx->launches = 0;
    cudaStream_t st = nullptr;
    g2_opts o2{};
    if (opts) o2 = *opts;
    if (o2.work_bytes) o2.flags |= G2_FLAG_WORK_MODEL;
    TaskList tl;
    int rc = prepare_tasks(ctx, sources, nsrc, false, &o2, match_warps(ctx, &o2), st, &tl, false);
    if (rc) return rc;
    if (!sources) nsrc = ctx->n;
    ctx->last_split = tl.split;
    ctx->last_cap = tl.cap;
    rc = prepare_root_outputs(ctx, o2.root_nodes != nullptr, o2.root_cost != nullptr, st);
    if (!rc) rc = grow(ctx, ctx->d_out, ctx->out_cap, 1, "out");
    if (!rc)
        rc = match_enqueue(ctx, tl, &o2, ctx->d_out, o2.root_nodes ? ctx->d_root_nodes : nullptr,
                           o2.root_cost ? ctx->d_root_cost : nullptr, st);
    if (rc) return rc;
    unsigned long long h = 0;
    int status = 0;
    G2_TRY(cudaMemcpy(&h, ctx->d_out, sizeof(h), cudaMemcpyDeviceToHost));
    G2_TRY(cudaMemcpy(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    *count = h;
    if (o2.work_bytes) {
        rc = g2_last_work_bytes(ctx, o2.work_bytes);
        if (rc) return rc;
    }
    rc = gather_root_outputs(ctx, sources, nsrc, o2.root_nodes, o2.root_cost);
    if (rc) return rc;
    return status_to_code(status);
}

// ---------------------------------------------------------- batches of graphs

int g2_batch_load(g2_ctx *ctx, const g2_batch_graph *graphs, uint32_t ngraphs) {
    if (!ctx || (!graphs && ngraphs) || ngraphs > kMaxBatchGraphs) return G2_ERR_INVALID;
    uint64_t n = 0, m = 0;
    bool cores = ngraphs > 0;
    for (uint32_t g = 0; g < ngraphs; g++) {
        const g2_batch_graph &b = graphs[g];
        if (!b.row_ptrs || (!b.cols && b.m) || b.row_ptrs[b.n] != b.m) return G2_ERR_INVALID;
        n += b.n;
        m += b.m;
        cores = cores && b.core;
    }
    if (n >= (1ull << 32)) return G2_ERR_INVALID;
    // the disjoint union: graph g's vertices are shifted by the vertices before it
    std::vector<uint64_t> rp(n + 1), off(ngraphs + 1);
    std::vector<uint32_t> ci(m ? m : 1), core(cores ? n : 0);
    uint64_t v0 = 0, e0 = 0;
    for (uint32_t g = 0; g < ngraphs; g++) {
        const g2_batch_graph &b = graphs[g];
        off[g] = v0;
        for (uint64_t i = 0; i < b.n; i++) rp[v0 + i] = e0 + b.row_ptrs[i];
        for (uint64_t e = 0; e < b.m; e++) ci[e0 + e] = (uint32_t)(v0 + b.cols[e]);
        if (cores) std::copy(b.core, b.core + b.n, core.begin() + v0);
        v0 += b.n;
        e0 += b.m;
    }
    rp[n] = m;
    off[ngraphs] = n;
    int rc = g2_load_csr(ctx, rp.data(), ci.data(), n, m);
    if (!rc && cores) rc = g2_load_core(ctx, core.data());
    if (!rc) rc = grow(ctx, ctx->d_goff, ctx->goff_cap, ngraphs + 1, "batch offsets");
    if (rc) return rc;
    G2_TRY(cudaMemcpy(ctx->d_goff, off.data(), sizeof(uint64_t) * (ngraphs + 1), cudaMemcpyHostToDevice));
    ctx->batch_off = off;
    return G2_OK;
}

// Per-graph sums of the per-task counts of the last run into host `counts`.
static int batch_counts(g2_ctx *ctx, const uint64_t *d_per_task, uint64_t *counts, cudaStream_t st) {
    const uint32_t ng = (uint32_t)ctx->batch_off.size() - 1;
    int rc = grow(ctx, ctx->d_gcount, ctx->gcount_cap, ng, "batch counts");
    if (rc) return rc;
    G2_TRY(cudaMemsetAsync(ctx->d_gcount, 0, sizeof(unsigned long long) * ng, st));
    segment_sum_kernel<<<ctx->sm_count * 2, 512, 0, st>>>(ctx->d_tasks, d_per_task, ctx->last_cap,
                                                          ctx->last_split ? ctx->d_ntask : nullptr, ctx->d_goff, ng,
                                                          ctx->d_gcount);
    ctx->launches++;
    G2_TRY(cudaMemcpyAsync(counts, ctx->d_gcount, sizeof(uint64_t) * ng, cudaMemcpyDeviceToHost, st));
    G2_TRY(cudaStreamSynchronize(st));
    return G2_OK;
}

int g2_batch_mce(g2_ctx *ctx, const g2_opts *opts, uint64_t *counts, uint64_t *hist, uint32_t hist_len) {
    if (!ctx || !counts || (hist && hist_len == 0)) return G2_ERR_INVALID;
    if (ctx->batch_off.size() < 2) return G2_ERR_NO_GRAPH;
    G2_TRY(cudaSetDevice(ctx->device));
    ctx->launches = 0;
    const uint32_t hl = hist ? hist_len : 0u;
    cudaStream_t st = nullptr;
    g2_opts o2{};
    if (opts) o2 = *opts;
    o2.root_nodes = o2.root_cost = nullptr;
    o2.work_bytes = nullptr;
    o2.flags &= ~G2_FLAG_WORK_MODEL;
    TaskList tl;
    int rc = prepare_tasks(ctx, nullptr, 0, false, &o2, mce_warps(ctx, &o2), st, &tl, true);
    if (rc) return rc;
    ctx->last_split = tl.split;
    ctx->last_cap = tl.cap;
    rc = grow(ctx, ctx->d_root_cliques, ctx->root_cliques_cap, ctx->tasks_cap, "root cliques");
    if (!rc) rc = grow(ctx, ctx->d_out, ctx->out_cap, 1 + hl, "out");
    if (rc) return rc;
    G2_TRY(cudaMemsetAsync(ctx->d_root_cliques, 0, sizeof(uint64_t) * ctx->tasks_cap, st));
    rc = mce_enqueue(ctx, tl, &o2, ctx->d_out, hl, nullptr, nullptr, st, ctx->d_root_cliques);
    if (!rc) rc = mce_host_spill(ctx, st);
    if (!rc) rc = batch_counts(ctx, ctx->d_root_cliques, counts, st);
    if (rc) return rc;
    std::vector<unsigned long long> h(1 + hl);
    int status = 0;
    G2_TRY(cudaMemcpy(h.data(), ctx->d_out, sizeof(unsigned long long) * (1 + hl), cudaMemcpyDeviceToHost));
    G2_TRY(cudaMemcpy(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (hist)
        for (uint32_t s = 0; s < hist_len; s++) hist[s] = h[1 + s];
    return status_to_code(status);
}

int g2_batch_match(g2_ctx *ctx, const g2_opts *opts, uint64_t *counts) {
    if (!ctx || !counts) return G2_ERR_INVALID;
    if (ctx->batch_off.size() < 2) return G2_ERR_NO_GRAPH;
    if (!ctx->has_plan) return G2_ERR_NO_PLAN;
    G2_TRY(cudaSetDevice(ctx->device));
    ctx->launches = 0;
    cudaStream_t st = nullptr;
    g2_opts o2{};
    if (opts) o2 = *opts;
    o2.root_nodes = o2.root_cost = nullptr;
    o2.work_bytes = nullptr;
    o2.flags &= ~G2_FLAG_WORK_MODEL;
    TaskList tl;
    int rc = prepare_tasks(ctx, nullptr, 0, false, &o2, match_warps(ctx, &o2), st, &tl, false);
    if (rc) return rc;
    ctx->last_split = tl.split;
    ctx->last_cap = tl.cap;
    rc = prepare_root_outputs(ctx, true, false, st);  // per-task counts
    if (!rc) rc = grow(ctx, ctx->d_out, ctx->out_cap, 1, "out");
    if (!rc) rc = match_enqueue(ctx, tl, &o2, ctx->d_out, ctx->d_root_nodes, nullptr, st);
    if (!rc) rc = batch_counts(ctx, ctx->d_root_nodes, counts, st);
    if (rc) return rc;
    int status = 0;
    G2_TRY(cudaMemcpy(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost));
    return status_to_code(status);
}

// ---------------------------------------------------------- cost model

int g2_root_features(g2_ctx *ctx, const uint32_t *sources, uint64_t nsrc, float *out) {
    if (!ctx || !out) return G2_ERR_INVALID;
    if (!ctx->d_rp) return G2_ERR_NO_GRAPH;
    G2_TRY(cudaSetDevice(ctx->device));
    if (!sources) nsrc = ctx->n;
    uint32_t *d_src = nullptr;
    float *d_f = nullptr;
    if (sources) G2_TRY(cudaMalloc(&d_src, sizeof(uint32_t) * std::max<uint64_t>(nsrc, 1)));
    cudaError_t e = cudaMalloc(&d_f, sizeof(float) * G2_MODEL_FEATURES * std::max<uint64_t>(nsrc, 1));
    if (e == cudaSuccess && sources)
        e = cudaMemcpy(d_src, sources, sizeof(uint32_t) * nsrc, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nsrc)
        e = g2::features_launch(ctx->d_rp, ctx->d_ci, ctx->d_fo, core_of(ctx), d_src, nsrc, d_f, ctx->sm_count, 0);
    if (e == cudaSuccess)
        e = cudaMemcpy(out, d_f, sizeof(float) * G2_MODEL_FEATURES * nsrc, cudaMemcpyDeviceToHost);
    cudaFree(d_src);
    cudaFree(d_f);
    if (e != cudaSuccess) return fail_cuda(ctx, e, "g2_root_features");
    return G2_OK;
}

// Scratch of one training / gradient call, freed on return.
struct TrainBufs {
    float *X = nullptr, *Y = nullptr, *params = nullptr, *norm = nullptr, *grad = nullptr, *mom = nullptr,
          *vel = nullptr, *loss = nullptr;
    uint32_t *idx = nullptr;
    ~TrainBufs() {
        void *b[] = {X, Y, params, norm, grad, mom, vel, loss, idx};
        for (void *p : b)
            if (p) cudaFree(p);
    }
};

static int upload_train(g2_ctx *ctx, TrainBufs &b, const float *X, const float *Y, uint64_t n, const float *norm,
                        const float *params) {
    const uint64_t nn = std::max<uint64_t>(n, 1);
    G2_TRY(cudaMalloc(&b.X, sizeof(float) * G2_MODEL_FEATURES * nn));
    G2_TRY(cudaMalloc(&b.Y, sizeof(float) * nn));
    G2_TRY(cudaMalloc(&b.idx, sizeof(uint32_t) * nn));
    G2_TRY(cudaMalloc(&b.params, sizeof(float) * G2_MODEL_PARAMS));
    G2_TRY(cudaMalloc(&b.norm, sizeof(float) * G2_MODEL_NORM));
    G2_TRY(cudaMalloc(&b.grad, sizeof(float) * G2_MODEL_PARAMS));
    G2_TRY(cudaMalloc(&b.loss, sizeof(float)));
    G2_TRY(cudaMemcpy(b.X, X, sizeof(float) * G2_MODEL_FEATURES * n, cudaMemcpyHostToDevice));
    G2_TRY(cudaMemcpy(b.Y, Y, sizeof(float) * n, cudaMemcpyHostToDevice));
    G2_TRY(cudaMemcpy(b.params, params, sizeof(float) * G2_MODEL_PARAMS, cudaMemcpyHostToDevice));
    G2_TRY(cudaMemcpy(b.norm, norm, sizeof(float) * G2_MODEL_NORM, cudaMemcpyHostToDevice));
    return G2_OK;
}

int g2_model_grad(g2_ctx *ctx, const float *X, const float *y, uint32_t n, const float *norm, const float *params,
                  float *grad, float *loss) {
    if (!ctx || !X || !y || !norm || !params || !grad || n == 0) return G2_ERR_INVALID;
    G2_TRY(cudaSetDevice(ctx->device));
    TrainBufs b;
    int rc = upload_train(ctx, b, X, y, n, norm, params);
    if (rc) return rc;
    std::vector<uint32_t> idx(n);
    std::iota(idx.begin(), idx.end(), 0u);
    G2_TRY(cudaMemcpy(b.idx, idx.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
    G2_TRY(cudaMemset(b.grad, 0, sizeof(float) * G2_MODEL_PARAMS));
    G2_TRY(cudaMemset(b.loss, 0, sizeof(float)));
    G2_TRY(g2::train_step_launch(b.X, b.Y, b.idx, n, b.params, b.norm, b.grad, b.loss, 0));
    G2_TRY(cudaMemcpy(grad, b.grad, sizeof(float) * G2_MODEL_PARAMS, cudaMemcpyDeviceToHost));
    float l = 0.f;
    G2_TRY(cudaMemcpy(&l, b.loss, sizeof(float), cudaMemcpyDeviceToHost));
    if (loss) *loss = l / (float)n;
    return G2_OK;
}

int g2_model_train(g2_ctx *ctx, const float *X, const float *cost, uint64_t n, uint32_t epochs, uint32_t batch,
                   float lr, uint64_t seed, float *params, float *norm, float *epoch_loss) {
    if (!ctx || !X || !cost || !params || !norm || n < 2 || n >= (1ull << 31) || batch == 0) return G2_ERR_INVALID;
    G2_TRY(cudaSetDevice(ctx->device));
    const int F = G2_MODEL_FEATURES;
    // normalisation of features and of the log-cost targets
    std::vector<double> mean(F, 0.0), var(F, 0.0);
    std::vector<float> y(n);
    double ym = 0.0, yv = 0.0;
    for (uint64_t i = 0; i < n; i++) {
        for (int k = 0; k < F; k++) mean[k] += X[i * F + k];
        y[i] = std::log1p(std::max(0.f, cost[i]));
        ym += y[i];
    }
    for (int k = 0; k < F; k++) mean[k] /= (double)n;
    ym /= (double)n;
    for (uint64_t i = 0; i < n; i++) {
        for (int k = 0; k < F; k++) var[k] += (X[i * F + k] - mean[k]) * (X[i * F + k] - mean[k]);
        yv += (y[i] - ym) * (y[i] - ym);
    }
    for (int k = 0; k < F; k++) {
        norm[k] = (float)mean[k];
        norm[F + k] = (float)std::max(1e-3, std::sqrt(var[k] / (double)n));
    }
    norm[2 * F] = (float)ym;
    norm[2 * F + 1] = (float)std::max(1e-3, std::sqrt(yv / (double)n));
    for (uint64_t i = 0; i < n; i++) y[i] = (y[i] - norm[2 * F]) / norm[2 * F + 1];
    // He-uniform initialisation
    std::mt19937_64 rng(seed);
    auto uni = [&](float lim) { return std::uniform_real_distribution<float>(-lim, lim)(rng); };
    for (int i = 0; i < 64 * F; i++) params[i] = uni(std::sqrt(6.f / F));
    for (int i = 0; i < 64; i++) params[64 * F + i] = 0.f;
    for (int i = 0; i < 64 * 64; i++) params[64 * F + 64 + i] = uni(std::sqrt(6.f / 64));
    for (int i = 0; i < 64; i++) params[64 * F + 64 + 4096 + i] = 0.f;
    for (int i = 0; i < 64; i++) params[64 * F + 128 + 4096 + i] = uni(std::sqrt(6.f / 64));
    params[G2_MODEL_PARAMS - 1] = 0.f;
    TrainBufs b;
    int rc = upload_train(ctx, b, X, y.data(), n, norm, params);
    if (rc) return rc;
    G2_TRY(cudaMalloc(&b.mom, sizeof(float) * G2_MODEL_PARAMS));
    G2_TRY(cudaMalloc(&b.vel, sizeof(float) * G2_MODEL_PARAMS));
    G2_TRY(cudaMemset(b.mom, 0, sizeof(float) * G2_MODEL_PARAMS));
    G2_TRY(cudaMemset(b.vel, 0, sizeof(float) * G2_MODEL_PARAMS));
    std::vector<uint32_t> perm(n);
    std::iota(perm.begin(), perm.end(), 0u);
    int step = 0;
    for (uint32_t ep = 0; ep < epochs; ep++) {
        std::shuffle(perm.begin(), perm.end(), rng);
        G2_TRY(cudaMemcpy(b.idx, perm.data(), sizeof(uint32_t) * n, cudaMemcpyHostToDevice));
        G2_TRY(cudaMemset(b.loss, 0, sizeof(float)));
        for (uint64_t s = 0; s < n; s += batch) {
            const uint32_t m = (uint32_t)std::min<uint64_t>(batch, n - s);
            G2_TRY(cudaMemsetAsync(b.grad, 0, sizeof(float) * G2_MODEL_PARAMS));
            G2_TRY(g2::train_step_launch(b.X, b.Y, b.idx + s, m, b.params, b.norm, b.grad, b.loss, 0));
            G2_TRY(g2::adam_launch(b.params, b.mom, b.vel, b.grad, lr, ++step, 0));
        }
        if (epoch_loss) {
            float l = 0.f;
            G2_TRY(cudaMemcpy(&l, b.loss, sizeof(float), cudaMemcpyDeviceToHost));
            epoch_loss[ep] = l / (float)n;
        }
    }
    G2_TRY(cudaMemcpy(params, b.params, sizeof(float) * G2_MODEL_PARAMS, cudaMemcpyDeviceToHost));
    // Calibration of the decoded cost: a least-squares fit in log space shrinks
    // the spread of its predictions, which shrinks exactly the heavy roots that
    // splitting must see.  Rescale the decode so that the predictions on the
    // training set have the targets' mean and spread (variance matching).
    {
        float *d_pred = nullptr;
        G2_TRY(cudaMalloc(&d_pred, sizeof(float) * n));
        cudaError_t e = g2::score_launch(nullptr, nullptr, nullptr, nullptr, nullptr, n, b.X, b.params, b.norm,
                                         d_pred, nullptr, nullptr, ctx->sm_count, 0);
        std::vector<float> pred(n);
        if (e == cudaSuccess) e = cudaMemcpy(pred.data(), d_pred, sizeof(float) * n, cudaMemcpyDeviceToHost);
        cudaFree(d_pred);
        if (e != cudaSuccess) return fail_cuda(ctx, e, "calibration");
        double pm = 0.0, pv = 0.0;
        for (float p : pred) pm += p;
        pm /= (double)n;
        for (float p : pred) pv += (p - pm) * (p - pm);
        const double ps = std::sqrt(pv / (double)n);
        if (ps > 1e-3) {  // decode(y) = y * ystd' + ymean' with (y - pm) / ps rescaled to unit spread
            const double ystd = norm[2 * F + 1], ymean = norm[2 * F];
            norm[2 * F + 1] = (float)(ystd / ps);
            norm[2 * F] = (float)(ymean - pm * ystd / ps);
        }
    }
    return G2_OK;
}

int g2_model_predict(g2_ctx *ctx, const float *X, uint64_t n, const float *norm, const float *params, float *out) {
    if (!ctx || !X || !norm || !params || !out) return G2_ERR_INVALID;
    G2_TRY(cudaSetDevice(ctx->device));
    if (n == 0) return G2_OK;
    TrainBufs b;
    int rc = upload_train(ctx, b, X, X, 0, norm, params);  // X / params / norm only
    if (rc) return rc;
    float *d_x = nullptr, *d_p = nullptr;
    G2_TRY(cudaMalloc(&d_x, sizeof(float) * G2_MODEL_FEATURES * n));
    cudaError_t e = cudaMalloc(&d_p, sizeof(float) * n);
    if (e == cudaSuccess) e = cudaMemcpy(d_x, X, sizeof(float) * G2_MODEL_FEATURES * n, cudaMemcpyHostToDevice);
    if (e == cudaSuccess)
        e = g2::score_launch(nullptr, nullptr, nullptr, nullptr, nullptr, n, d_x, b.params, b.norm, d_p, nullptr,
                             nullptr, ctx->sm_count, 0);
    if (e == cudaSuccess) e = cudaMemcpy(out, d_p, sizeof(float) * n, cudaMemcpyDeviceToHost);
    cudaFree(d_x);
    cudaFree(d_p);
    if (e != cudaSuccess) return fail_cuda(ctx, e, "g2_model_predict");
    return G2_OK;
}

int g2_set_model(g2_ctx *ctx, const float *params, const float *norm) {
    if (!ctx || !params || !norm) return G2_ERR_INVALID;
    G2_TRY(cudaSetDevice(ctx->device));
    if (!ctx->d_model) G2_TRY(cudaMalloc(&ctx->d_model, sizeof(float) * (G2_MODEL_PARAMS + G2_MODEL_NORM)));
    G2_TRY(cudaMemcpy(ctx->d_model, params, sizeof(float) * G2_MODEL_PARAMS, cudaMemcpyHostToDevice));
    G2_TRY(cudaMemcpy(ctx->d_model + G2_MODEL_PARAMS, norm, sizeof(float) * G2_MODEL_NORM, cudaMemcpyHostToDevice));
    return G2_OK;
}

}  // extern "C"

namespace g2rt {
int g2_after_load(g2_ctx *ctx) { return after_load(ctx); }
}  // namespace g2rt
