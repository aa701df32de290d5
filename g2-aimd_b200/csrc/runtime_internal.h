// runtime_internal.h - the context behind the C ABI and the enqueue helpers
// shared by the translation units of libg2aimd.so (runtime.cu, view_run.cu).
// Not installed: callers see only include/g2_aimd.h.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <string>
#include <utility>
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
    uint32_t max_fwd = 0;      // max |N(v) ∩ (v, ∞)|
    uint32_t *d_fo = nullptr;  // forward-list offsets
    uint64_t fo_cap = 0;
    uint32_t *d_core = nullptr;  // optional core numbers (cost-model feature)
    bool core_loaded = false;    // d_core holds the loaded graph's core numbers
    uint64_t rp_cap = 0, ci_cap = 0;       // owned CSR buffers (entries), reused by later loads
    unsigned int *d_fwdmax = nullptr;      // max forward degree of a load
    uint64_t core_cap = 0;
    // work buffers
    uint32_t *d_scratch = nullptr;
    uint64_t scratch_words = 0;
    uint32_t *d_tasks = nullptr;  // root vertex per task (schedule order)
    uint32_t *d_defer = nullptr;  // 3 deferred lists of tasks_cap each
    uint64_t tasks_cap = 0;
    uint64_t *d_root_nodes = nullptr, *d_root_cost = nullptr;
    uint64_t root_nodes_cap = 0, root_cost_cap = 0;
    unsigned long long *d_ctr = nullptr;  // kCtr* layout below
    uint32_t *d_rec = nullptr;            // MCE hand-off records
    uint32_t *d_ready = nullptr;          // their ready words
    uint32_t *d_epoch = nullptr;          // epoch of the current run (bumped on the device)
    uint32_t *d_pool = nullptr;           // MCE spill row pool
    int *d_status = nullptr;
    unsigned long long *d_deadline = nullptr;  // %globaltimer ns of a run's time budget
    unsigned long long *d_out = nullptr;  // counters for the host entry points
    uint64_t out_cap = 0;
    // schedule
    uint64_t *d_keys = nullptr, *d_keys2 = nullptr;
    uint64_t keys_cap = 0, keys2_cap = 0;
    uint32_t *d_roots = nullptr, *d_S = nullptr, *d_part = nullptr, *d_xroots = nullptr, *d_xparts = nullptr;
    uint64_t roots_cap = 0, S_cap = 0, part_cap = 0, xroots_cap = 0, xparts_cap = 0;
    float *d_cost = nullptr, *d_total = nullptr;
    uint64_t cost_cap = 0, total_cap = 0;
    unsigned long long *d_ntask = nullptr;
    uint64_t ntask_cap = 0;
    void *d_cub = nullptr;
    size_t cub_bytes = 0;
    bool last_split = false;  // the last run's tasks carry parts
    uint64_t last_cap = 0;    // tasks buffer entries used by the last run
    // learned cost model: params (G2_MODEL_PARAMS) followed by norm (G2_MODEL_NORM)
    float *d_model = nullptr;
    float *d_feat = nullptr;  // per-vertex features of the loaded graph (n x 8), cached
    uint64_t feat_cap = 0;
    bool feat_valid = false;
    // plan
    g2::DevPlan plan{};
    bool has_plan = false;
    bool clique_plan = false;
    // diagnostics
    std::string cuda_err;
    uint64_t launches = 0;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};  // around the enumeration passes
    g2::MceArgs last_mce{};            // arguments of the last MCE enqueue (host-spill pass)
    int last_mce_wpl = 1;
    uint64_t host_spill_bytes = 1ull << 30;  // managed slab for roots no device slab holds
    void *h_spill = nullptr;
    uint64_t h_spill_bytes = 0;
    // batch of graphs loaded as one disjoint union (g2_batch_load)
    std::vector<uint64_t> batch_off;  // first vertex of each graph, then n
    uint64_t *d_goff = nullptr;
    uint64_t goff_cap = 0;
    uint64_t *d_root_cliques = nullptr;
    uint64_t root_cliques_cap = 0;
    unsigned long long *d_gcount = nullptr;
    uint64_t gcount_cap = 0;
    // out-of-core view runs: pinned host slots and the two device slots, kept
    // between calls (pinning and device allocation stall other CUDA calls)
    std::vector<std::pair<void *, uint64_t>> view_host;
    void *view_dev[2] = {nullptr, nullptr};
    void *view_builder = nullptr;  // g2rt::DeviceViewBuilder kept between view runs (its work arrays)
    uint64_t view_dev_cap[2] = {0, 0};
    bool timed = false;
    int timed_passes = 0;  // enumeration passes the last timed run recorded (MCE 3, match 1)
    unsigned long long *d_work = nullptr;
    cudaStream_t last_stream = nullptr;
};

namespace g2rt {

// Record a CUDA error in the context; G2_ERR_OOM for allocation failures.
int fail_cuda(g2_ctx *c, cudaError_t e, const char *where);
// Per-graph set-up after a new CSR is in the context (forward offsets, ...).
int g2_after_load(g2_ctx *ctx);
// Release a context's device view builder (view_device.cu).
void view_builder_free(void *builder);
int fail_cuda_if(g2_ctx *c, cudaError_t e, const char *where);

#define G2_TRY(call)                                             \
    do {                                                         \
        cudaError_t _e = (call);                                 \
        if (_e != cudaSuccess) return fail_cuda(ctx, _e, #call); \
    } while (0)

// Grow a device buffer to `need` entries (contents are not kept).
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

struct TaskList {
    uint64_t cap = 0;    // d_tasks entries in use (upper bound of the task count)
    bool split = false;  // d_part valid; the task count is in d_ntask
};

// Task generation on `st` (sources on the host or, with on_device, the device).
int prepare_tasks(g2_ctx *ctx, const uint32_t *sources, uint64_t nsrc, bool on_device, const g2_opts *o,
                  uint64_t nwarps, cudaStream_t st, TaskList *tl, bool mce);
// The enumeration passes of one run, enqueued on `st`.
int mce_enqueue(g2_ctx *ctx, const TaskList &tl, const g2_opts *o, unsigned long long *d_out, uint32_t hist_len,
                uint64_t *d_root_nodes, uint64_t *d_root_cost, cudaStream_t st, uint64_t *d_root_cliques = nullptr);
int match_enqueue(g2_ctx *ctx, const TaskList &tl, const g2_opts *o, unsigned long long *d_out,
                  uint64_t *d_root_nodes, uint64_t *d_root_cost, cudaStream_t st);
// After a synchronous MCE run: roots no device slab held, on the managed spill slab.
int mce_host_spill(g2_ctx *ctx, cudaStream_t st);
// Device-stream MCE runs: the same pass in stream order, then a flag for entries left.
int mce_stream_spill(g2_ctx *ctx, cudaStream_t st);
// Resident warps of the persistent grids (split targets).
uint64_t mce_warps(g2_ctx *ctx, const g2_opts *o);
uint64_t match_warps(g2_ctx *ctx, const g2_opts *o);
// Device status word -> G2_ERR_*.
int status_to_code(int st);

}  // namespace g2rt
