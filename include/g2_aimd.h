/*
 * g2_aimd.h - C ABI of the B200 subgraph-search library (libg2aimd.so).
 *
 * The reference (lyuheng/g2-aimd) exposes its hot path as a compile-time C++
 * template plugin: Worker<App>::run (system/worker.h:28) builds a
 * PipelineExecutor<App> (system/pipeline_executor.h:44), which uploads one CSR
 * view bin (Transfer, system/pipeline_executor.h:121-147), runs the BFS level
 * loop (Run, system/pipeline_executor.h:151-207) and reads the app's counters
 * (BK: totalCliques, app_BK/BK.h:38-76; GMatch: total_counts_ summed in
 * system/worker.h:250-279).  This header replaces that plugin boundary with plain
 * functions over plain pointers: one context per device, a CSR upload, a
 * query-plan upload and one call per enumeration.  Every call returns an int
 * status (0 = G2_OK, negative = error; see g2_strerror), outputs are
 * caller-owned, and no call exits the process (the reference prints and calls
 * exit(-1), common/gpu_env.h:85-92).
 *
 * Types follow the reference .bin format (common/graph.h:360-398):
 * vertex ids uint32_t (uintV, common/meta.h:15), edge offsets uint64_t (uintE,
 * common/meta.h:16); neighbour lists sorted, deduplicated, no self loops,
 * every edge stored in both directions.
 */
#ifndef G2_AIMD_H
#define G2_AIMD_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define G2_OK 0
#define G2_ERR_INVALID (-1)      /* bad argument (null pointer, size, range)  */
#define G2_ERR_CUDA (-2)         /* CUDA runtime error; see g2_last_cuda_error */
#define G2_ERR_OOM (-3)          /* device or pinned allocation failed         */
#define G2_ERR_TIMEOUT (-4)      /* a bounded device wait ran out (hang guard) */
#define G2_ERR_OVERFLOW (-5)     /* scratch and host spill both exhausted      */
#define G2_ERR_NO_GRAPH (-6)     /* no CSR loaded in this context              */
#define G2_ERR_NO_PLAN (-7)      /* g2_match_run without g2_set_plan           */
#define G2_ERR_UNSUPPORTED (-8)  /* e.g. query larger than G2_MAX_QUERY        */
#define G2_ERR_IO (-9)           /* file could not be read or written          */
#define G2_ERR_HIST (-10)        /* clique larger than the histogram supplied  */
#define G2_ERR_DEADLINE (-11)    /* g2_opts.deadline_ms ran out: the outputs hold
                                    the roots that finished (per-root outputs of
                                    the others stay 0)                          */

/* Largest query pattern: the reference keeps a partial embedding in
 * partial_subgraphs[WARPS_EACH_BLK][8] (app_gmatch/gmatch.h:87). */
#define G2_MAX_QUERY 8

/* Condition operators, same values as CondOperator (common/meta.h:22). */
#define G2_COND_LESS_THAN 0
#define G2_COND_LARGER_THAN 1
#define G2_COND_NON_EQUAL 2

/* Store strategies, same values as StoreStrategy (common/meta.h:24). */
#define G2_STORE_EXPAND 0
#define G2_STORE_PREFIX 1
#define G2_STORE_COUNT 2

/*
 * Query plan: the flat arrays of GMContext (system/appbase.h:11-68) as built by
 * Plan (system/plan.h:51-372) and uploaded by AppBase::allocateGMMemory
 * (system/appbase.h:156-216), with fixed capacity G2_MAX_QUERY.
 * Indexing follows the reference exactly:
 *   - by POSITION p in the match order: bn_*, pre_bn_*, after_bn_*, share,
 *     strategy (strategy has k+1 entries, strategy[k] = COUNT);
 *   - by QUERY VERTEX u: cond_*, pre_cond_*, after_cond_*;
 *   - entries of bn / cond lists are QUERY VERTEX ids (map with id2order).
 * cond[u][j] = {op, query vertex}: LESS_THAN means M(u) < M(vertex).
 */
typedef struct g2_plan {
    uint32_t k;                                   /* query vertices          */
    uint32_t hop;                                 /* Plan::GetHop            */
    uint32_t root_degree;                         /* Plan::root_degree_      */
    uint32_t order[G2_MAX_QUERY];                 /* matchOrder (seq_)       */
    uint32_t id2order[G2_MAX_QUERY];              /* ID2order (reverse_seq_) */
    uint32_t bn_count[G2_MAX_QUERY];
    uint32_t bn[G2_MAX_QUERY][G2_MAX_QUERY];
    uint32_t parent[G2_MAX_QUERY];                /* parentHost (unused on device) */
    uint32_t cond_count[G2_MAX_QUERY];
    uint32_t cond[G2_MAX_QUERY][G2_MAX_QUERY][2];
    uint32_t share[G2_MAX_QUERY];                 /* shareIntersection (0/1) */
    uint32_t pre_bn_count[G2_MAX_QUERY];
    uint32_t pre_bn[G2_MAX_QUERY][G2_MAX_QUERY];
    uint32_t pre_cond_count[G2_MAX_QUERY];
    uint32_t pre_cond[G2_MAX_QUERY][G2_MAX_QUERY][2];
    uint32_t after_bn_count[G2_MAX_QUERY];
    uint32_t after_bn[G2_MAX_QUERY][G2_MAX_QUERY];
    uint32_t after_cond_count[G2_MAX_QUERY];
    uint32_t after_cond[G2_MAX_QUERY][G2_MAX_QUERY][2];
    uint32_t strategy[G2_MAX_QUERY + 1];
    uint32_t moving_lvl[G2_MAX_QUERY];
} g2_plan;

/* Root schedule (task order of the device work queue). */
#define G2_SCHED_GIVEN 0      /* sources in the order given                      */
#define G2_SCHED_HEURISTIC 1  /* plain heuristic: descending forward degree x core */
#define G2_SCHED_SCORES 2     /* descending caller scores                          */
#define G2_SCHED_LEARNED 3    /* descending cost predicted on the device by the model
                                 set with g2_set_model (features + MLP fused into
                                 task generation); GMatch splits heavy roots by
                                 default                                          */

/*
 * Run options.  Zero-initialise and set what you need; 0 means "default".
 */
typedef struct g2_opts {
    uint32_t blocks;            /* persistent CTAs (default: 148 x occupancy)       */
    uint32_t warps_per_block;   /* default 8                                        */
    uint32_t schedule;          /* G2_SCHED_*                                       */
    uint32_t split_granularity; /* heavy-root splits aim at tasks of cost
                                   total / (granularity x warps) (0 = 4)           */
    const float *scores;        /* host, nsrc entries, for G2_SCHED_SCORES          */
    uint64_t *root_nodes;       /* optional host out: search-tree nodes per source
                                   (MCE) or embeddings per source (match), summed
                                   over a source's split tasks                      */
    uint64_t *work_bytes;       /* optional host out: algorithmic bytes W (MCE)     */
    uint32_t intersect_mode;    /* GMatch: 0 auto (clique bitmap path when the plan is
                                   a clique), 1 generic plan-driven path only        */
    uint32_t flags;             /* G2_FLAG_* bits                                    */
    uint32_t split_depth;       /* MCE: a split root's tasks share out its subtrees
                                   at this search-tree depth (0 = default 2)         */
    uint64_t *root_cost;        /* optional host out: SM cycles per source (summed
                                   over its split tasks)                            */
    uint32_t chunk;             /* tasks taken per queue atomic (0 = 1 MCE, 4 match) */
    uint32_t spill_kcycles;     /* MCE and plan walks of non-clique plans: every this
                                   many thousand SM cycles a walk checks for idle
                                   warps and hands them the pending work of its
                                   shallowest open level (0 = 20)                   */
    uint32_t ctas_per_sm;       /* GMatch register budget, as CTAs of 256 threads per
                                   SM: 0 or 4 (64 registers), 6 (40 registers, more
                                   resident warps; pays on graphs larger than L2)   */
    uint32_t wait_cycles;       /* hang guard: the longest a warp waits for a handed-off
                                   record, in SM cycles (0 = 2^37, about 70 s); a run
                                   whose wait ran out returns G2_ERR_TIMEOUT and the
                                   context stays usable                             */
    uint32_t deadline_ms;       /* time budget of the run on the device (0 = none).
                                   Past it, warps start no new root and drop the root
                                   they are walking (nothing of it counted), so the
                                   run ends soon after; it returns G2_ERR_DEADLINE
                                   with the totals and per-root outputs of the roots
                                   that finished: MCE root_nodes > 0, match
                                   root_cost > 0 mark them.  Implies no hand-off.   */
} g2_opts;

/* g2_opts.flags */
#define G2_FLAG_TIME_KERNELS 1u  /* record CUDA events around each enumeration pass */
#define G2_FLAG_WORK_MODEL 2u    /* count the work model W on the device (slower)    */
#define G2_FLAG_SPLIT 4u         /* split heavy roots by the schedule's cost estimate:
                                    a root of estimated cost c becomes ceil(c / t)
                                    tasks (at most 256), t = total / (g x warps) with
                                    g = split_granularity; each task owns every k-th
                                    top-level branch of its root (GMatch) or every
                                    k-th subtree at depth split_depth (MCE)          */
#define G2_FLAG_NO_SPLIT 8u      /* GMatch G2_SCHED_LEARNED without splitting (MCE
                                    splits only with G2_FLAG_SPLIT; its walks hand
                                    branches to idle warps instead)                 */
#define G2_FLAG_NO_SPILL 16u     /* no hand-off of pending work to idle warps        */
#define G2_FLAG_L2_PERSIST 32u   /* device-stream runs: keep the tail of the column
                                    array (the dense core's adjacency) persisting in
                                    L2 during the enumeration launches               */

typedef struct g2_ctx g2_ctx;

/* Library version string and the text of an error code. */
const char *g2_version(void);
const char *g2_strerror(int code);
/* Text of the last CUDA error seen in this context (or "" if none). */
const char *g2_last_cuda_error(const g2_ctx *ctx);

/* Open a context on `device` (replaces the PipelineExecutor constructor,
 * system/pipeline_executor.h:44-99; no memory is pinned to "all free memory").
 * scratch_bytes = device scratch budget for DFS frames (0 = default 4 GiB). */
int g2_open(int device, uint64_t scratch_bytes, g2_ctx **out);
int g2_close(g2_ctx *ctx);

/* Upload a CSR from host memory (replaces Transfer,
 * system/pipeline_executor.h:121-147).  The context keeps a device copy. */
int g2_load_csr(g2_ctx *ctx, const uint64_t *row_ptrs, const uint32_t *cols,
                uint64_t n, uint64_t m);
/*
 * Batches of small graphs (C4-style workloads).  g2_batch_load loads the
 * graphs as one disjoint union (graph g's vertex i becomes off[g] + i), so one
 * launch per job covers every graph: a maximal clique or a connected pattern
 * lies inside one graph.  Per-graph results are summed on the device from the
 * per-root counts.  Ids inside each graph should be in degeneracy order.
 * At most 4096 graphs; the union must have fewer than 2^32 vertices.
 */
typedef struct g2_batch_graph {
    const uint64_t *row_ptrs;  /* n + 1 entries, host memory */
    const uint32_t *cols;      /* m entries */
    uint64_t n, m;
    const uint32_t *core;      /* optional core numbers (learned schedule); NULL in
                                  any graph means none are loaded */
} g2_batch_graph;

int g2_batch_load(g2_ctx *ctx, const g2_batch_graph *graphs, uint32_t ngraphs);
/* Maximal cliques per graph (counts[ngraphs]) and the size histogram of all. */
int g2_batch_mce(g2_ctx *ctx, const g2_opts *opts, uint64_t *counts, uint64_t *hist, uint32_t hist_len);
/* Matches of the plan set with g2_set_plan, per graph (counts[ngraphs]). */
int g2_batch_match(g2_ctx *ctx, const g2_opts *opts, uint64_t *counts);

/* Allocate the working buffers of runs over up to `max_sources` roots (0 = the
 * loaded graph's n): DFS slabs, counters, task lists and the MCE hand-off
 * record queue.  Optional; a run allocates what is missing.  Callers that time
 * runs separately from set-up (as the reference's workers allocate their
 * device buffers before the timed loop) call it once after loading. */
int g2_reserve(g2_ctx *ctx, uint64_t max_sources);

/* Borrow a CSR that already lives in device memory of this context's device.
 * The caller keeps it alive until the next load or g2_close. */
int g2_load_csr_device(g2_ctx *ctx, const uint64_t *d_row_ptrs,
                       const uint32_t *d_cols, uint64_t n, uint64_t m);

/* Upload a query plan (replaces AppBase::allocateGMMemory,
 * system/appbase.h:156-216). */
int g2_set_plan(g2_ctx *ctx, const g2_plan *plan);

/*
 * Maximal clique enumeration (Bron-Kerbosch with Tomita pivot) rooted at
 * `sources` (host array; NULL = every vertex 0..n-1).  Replaces app_BK
 * (BKExpandSequential, app_BK/BK.h:400-480) run through Worker/PipelineExecutor;
 * the result equals the sum of the reference's "Total No. of Cliques:" lines.
 * Root v starts with R={v}, P=N(v)∩(v,∞), X=N(v)∩[0,v) (app_BK/BK.h:323-355);
 * vertices without neighbours are skipped (app_BK/BK.h:335-336).
 * count: number of maximal cliques; hist[s] = maximal cliques with s vertices
 * (hist may be NULL; G2_ERR_HIST if a clique has >= hist_len vertices).
 */
int g2_mce_run(g2_ctx *ctx, const uint32_t *sources, uint64_t nsrc,
               const g2_opts *opts, uint64_t *count, uint64_t *hist,
               uint32_t hist_len);

/*
 * Plan-driven subgraph enumeration of the plan set by g2_set_plan, rooted at
 * `sources` (host array; NULL = all vertices).  Replaces GMatchApp
 * (app_gmatch/gmatch.h:15-736); *count equals the reference's "Total counts:"
 * line (system/worker.h:273-279): the number of embeddings that satisfy the
 * plan's symmetry-breaking conditions.
 */
int g2_match_run(g2_ctx *ctx, const uint32_t *sources, uint64_t nsrc,
                 const g2_opts *opts, uint64_t *count);

/*
 * Device-resident variants used for timing: sources and outputs live in device
 * memory of this context; work is enqueued on `stream` (a cudaStream_t, may be
 * NULL for the legacy default stream) and the call returns without
 * synchronising.  d_out receives the counters:
 *   MCE:   d_out[0] = count, d_out[1 + s] = hist[s] for s < hist_len;
 *   match: d_out[0] = count.
 * d_out must hold 1 + hist_len (MCE) or 1 (match) uint64_t.  The run's outcome
 * (what the synchronous entry point would return) is read with g2_run_status.
 */
int g2_mce_run_device(g2_ctx *ctx, const uint32_t *d_sources, uint64_t nsrc,
                      const g2_opts *opts, uint64_t *d_out, uint32_t hist_len,
                      void *stream);
int g2_match_run_device(g2_ctx *ctx, const uint32_t *d_sources, uint64_t nsrc,
                        const g2_opts *opts, uint64_t *d_out, void *stream);

/*
 * Outcome of the last device-stream run (g2_mce_run_device,
 * g2_match_run_device) of this context, enqueued on `stream`: waits for the
 * stream, then returns what the synchronous entry point would have returned:
 * G2_OK; G2_ERR_OVERFLOW (entries that no slab, spill slab included, held: the
 * counts leave them out); G2_ERR_TIMEOUT (a bounded device wait ran out);
 * G2_ERR_DEADLINE (the time budget ran out: the counts cover the roots that
 * finished); G2_ERR_HIST; G2_ERR_INVALID (inconsistent plan).  The status word
 * belongs to the context: the next run on it starts a new one.
 */
int g2_run_status(g2_ctx *ctx, void *stream);

/* Number of kernels the last run launched (for launch accounting). */
uint64_t g2_last_launch_count(const g2_ctx *ctx);

/* After a run with G2_FLAG_TIME_KERNELS: device milliseconds of enumeration
 * pass `pass` of the last run (MCE: 0 = main pass, 1-2 = deferred passes;
 * match: pass 0 only, G2_ERR_INVALID beyond), measured with CUDA events on the
 * run's stream.  Synchronises on the events. */
int g2_pass_time_ms(g2_ctx *ctx, int pass, float *ms);

/* After a run with G2_FLAG_WORK_MODEL: the work model W of the last run in
 * bytes (MCE: merge-intersection bytes of the reference's search tree; match:
 * 4 x sum over partial embeddings of the back neighbours' degrees).
 * Synchronises the run's stream. */
int g2_last_work_bytes(g2_ctx *ctx, uint64_t *bytes);

/* Degeneracy order of the loaded graph computed on the device (replaces the
 * host peeling of kmeans/kcore.cpp:39-191): perm[v] = new id of v, core[v] =
 * core number (optional).  Equal to g2_degeneracy_order's output. */
int g2_degeneracy_order_device(g2_ctx *ctx, uint32_t *perm, uint32_t *core);

/*
 * Out-of-core enumeration over view bins, for graphs whose CSR exceeds device
 * memory (replaces Worker::run's producer/consumer loop, system/worker.h:165-279,
 * with ViewBin::Materialize, view/view_bin.h:61-159, and
 * PipelineExecutor::Transfer, system/pipeline_executor.h:121-147).  The CSR
 * stays in host memory.  bin_of[v] is the bin of root v (G2_VIEW_NO_BIN: not a
 * root), as g2_read_vbmap or g2_view_bins give it.  Host threads build each
 * bin's view (g2_view_materialize) into pinned buffers; the context uploads
 * views into two device slots, the upload of the next view overlapping the
 * enumeration of the current one, and sums the per-bin results.  Every
 * maximal clique / match is found from exactly one root, so the totals equal
 * g2_mce_run / g2_match_run over the whole graph.  The context's loaded graph
 * is released (load again before other runs).  Per-root outputs, work model
 * and caller scores (G2_SCHED_SCORES) are not available here.
 */
#define G2_VIEW_NO_BIN 0xffffffffu
#define G2_VIEW_UPPER 1u     /* balls walked through vertices above their source */
#define G2_VIEW_FORWARD 4u   /* rows keep only neighbours above their own vertex */
#define G2_VIEW_EGO 8u       /* radius-1 views: rows keep only edges inside the ego network
                                N[s] of some root s of the bin (also a g2_view_opts flag) */
#define G2_VIEW_NO_UPPER 2u  /* g2_view_opts: full balls and rows even where the query
                                allows upper balls and forward rows; G2_VIEW_EGO there asks
                                for ego rows (radius-1 views only) */
#define G2_VIEW_DEVICE 16u   /* g2_view_opts: the GPU builds each view (same bytes as the
                                host build) straight into its device slot, reading the
                                host CSR through mapped pinned memory (registered for the
                                call if it is not pinned); radius-1 views without ego rows
                                (MCE, triangles, cliques), else G2_ERR_UNSUPPORTED.  No
                                host producers, no uploads                       */
typedef struct g2_view_opts {
    uint32_t producers;   /* host threads building views (0 = min(8, cores), fewer
                             if their marks, 4 bytes and a bit per vertex each,
                             would pass 32 GB); the host's threads, or
                             G2_HOST_THREADS, are shared out over the producers
                             for large views                                     */
    uint32_t radius;      /* ball radius (0 = from the query: 1 for MCE)         */
    uint32_t row_radius;  /* rows kept up to this distance (0 = from the query)  */
    uint32_t flags;       /* G2_VIEW_NO_UPPER, G2_VIEW_EGO, G2_VIEW_DEVICE        */
    uint32_t slots;       /* pinned host buffers holding built views, each as
                             large as the largest view (0 = producers + 2; at
                             least 2): bounds pinned memory, as the reference's
                             -qs holders do                                     */
} g2_view_opts;
typedef struct g2_view_stats {
    uint64_t bins;            /* views enumerated (bins with a root of enough degree) */
    uint64_t view_vertices;   /* sum over views                                   */
    uint64_t view_edges;      /* column entries, summed over views                */
    uint64_t h2d_bytes;       /* bytes uploaded                                   */
    uint64_t max_view_bytes;  /* largest view                                     */
    double build_ms;          /* host time building views, summed over threads    */
    double wait_ms;           /* time the device side waited for a view           */
    double total_ms;          /* wall time of the call                            */
    double copy_ms;           /* device time of the uploads (CUDA events)         */
    double run_ms;            /* device time of the runs, task set-up included    */
} g2_view_stats;
int g2_view_mce(g2_ctx *ctx, const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n,
                const uint32_t *bin_of, uint32_t nbins, const g2_view_opts *vopts,
                const g2_opts *opts, uint64_t *count, uint64_t *hist, uint32_t hist_len,
                uint64_t *bin_counts, g2_view_stats *stats);
/* Matches of the plan set with g2_set_plan (view shape from its query, as
 * g2_plan_view_radius gives it; roots of degree below the query root's degree
 * are skipped). */
int g2_view_match(g2_ctx *ctx, const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n,
                  const uint32_t *bin_of, uint32_t nbins, const g2_view_opts *vopts,
                  const g2_opts *opts, uint64_t *count, uint64_t *bin_counts,
                  g2_view_stats *stats);

/* Rename the loaded graph by its degeneracy order on the device (replaces
 * kmeans/kcore.cpp:39-191: peeling, degree sort inside each shell, recode):
 * afterwards the context holds the recoded CSR (rows sorted; equal to
 * g2_recode(g2_degeneracy_order)) and its core numbers under the new names, as
 * g2_load_core would load them.  perm[old] = new id and core[old] (optional host
 * outputs, n entries).  Rows are sorted in device calls of at most 2^30 entries
 * (environment G2_RECODE_CHUNK overrides); a longer row, or n >= 2^31 - 1, gives
 * G2_ERR_UNSUPPORTED.  Needs about twice the CSR's device memory meanwhile. */
int g2_degeneracy_recode_device(g2_ctx *ctx, uint32_t *perm, uint32_t *core);
/* Copy the loaded CSR back to host memory (row_ptrs: n + 1, cols: m entries). */
int g2_copy_csr(g2_ctx *ctx, uint64_t *row_ptrs, uint32_t *cols);

/* Size of the spill slab on which a synchronous MCE run (g2_mce_run,
 * g2_batch_mce) walks the roots that no slab of the context's scratch holds,
 * after the deferral passes: managed memory (default 1 GiB, allocated on first
 * need) whose pages live on the GPU while used and in host memory when device
 * memory runs out; 0 = none: such roots make the run return G2_ERR_OVERFLOW.
 * g2_mce_run_device enqueues the same pass in stream order, allocating the
 * slab on its first run since it cannot know the need (managed pages are only
 * placed when touched); under a CUDA graph capture a slab not yet allocated
 * means no pass.  g2_run_status reports the roots it could not hold. */
int g2_set_host_spill(g2_ctx *ctx, uint64_t bytes);

/* Search-tree nodes the last MCE run handed from long walks to idle warps
 * (records) and the bytes of root rows it moved to the record row pool.
 * Synchronises the run's stream. */
int g2_last_spill_stats(g2_ctx *ctx, uint64_t *records, uint64_t *pool_bytes);

/*
 * Plan-driven count that allocates no memory (no counterpart in the reference,
 * which allocates all of its buffers itself).  For callers that cannot let a
 * library call cudaMalloc / cudaFree: applications whose device memory is owned
 * by their own caching allocator or a fixed budget, and latency-critical code
 * where those calls may synchronise the device.  Counts the embeddings of `plan`
 * rooted at every vertex of the device-resident CSR (same result as
 * g2_match_run with sources = NULL) into *d_count (device memory), enqueued on
 * `stream` of the current device; the count is ready when the stream is.
 * Scratch is a file-scope device array of G2_NOALLOC_SCRATCH_BYTES that every
 * GPU loading this library holds until exit.  Limits: n <= G2_NOALLOC_MAX_VERTICES,
 * otherwise G2_ERR_UNSUPPORTED (also when the query leaves too little scratch
 * per warp).  All calls on a device share that array: calls that overlap on the
 * GPU race and must be serialised.  The plan is passed to the kernel as an
 * argument, so a call may overlap context match runs of other plans.  Every
 * call looks up the array's device address on the current device (no
 * allocation).  A failure found on the device (the kernel's status word set)
 * is reported in stream order: *d_count holds G2_NOALLOC_FAILED instead of a
 * count.
 */
#define G2_NOALLOC_SCRATCH_BYTES (32u << 20)
#define G2_NOALLOC_MAX_VERTICES (1u << 21)
#define G2_NOALLOC_FAILED 0xffffffffffffffffull
int g2_match_count_noalloc(const uint64_t *d_row_ptrs, const uint32_t *d_cols,
                           uint64_t n, uint64_t m, const g2_plan *plan,
                           uint64_t *d_count, void *stream);

/*
 * Learned root-cost model (no counterpart in the reference; it only orders and
 * splits root tasks).  MLP 8 -> 64 -> 64 -> 1 with ReLU, fp32 master weights,
 * bf16 tensor-core arithmetic with fp32 accumulation.  params (G2_MODEL_PARAMS
 * floats): W1[64][8], b1[64], W2[64][64], b2[64], w3[64], b3.  norm
 * (G2_MODEL_NORM floats): feature mean[8], feature std[8], target mean, target
 * std; targets are log1p(cost), cost = SM cycles of a root's search.
 */
#define G2_MODEL_FEATURES 8
#define G2_MODEL_PARAMS 4801
#define G2_MODEL_NORM 18
/* Core numbers (n entries, host) used by feature f1; without them p stands in. */
int g2_load_core(g2_ctx *ctx, const uint32_t *core);
/* Features of each source (host out, nsrc x 8; sources NULL = all vertices). */
int g2_root_features(g2_ctx *ctx, const uint32_t *sources, uint64_t nsrc, float *out);
/* Train on (X, cost): computes norm, initialises params from seed (He uniform)
 * and runs `epochs` of mini-batch Adam on the device.  epoch_loss (optional,
 * epochs entries) receives the mean squared error in normalised units.  The
 * target mean/std in norm are then recalibrated so that the decoded training
 * predictions have the targets' mean and spread in log space (the fit shrinks
 * the spread, and with it the heavy roots that splitting must see). */
int g2_model_train(g2_ctx *ctx, const float *X, const float *cost, uint64_t n, uint32_t epochs,
                   uint32_t batch, float lr, uint64_t seed, float *params, float *norm,
                   float *epoch_loss);
/* One forward+backward on (X, y_normalised) without updating: gradient of the
 * mean squared error w.r.t. params (G2_MODEL_PARAMS floats) and the loss. */
int g2_model_grad(g2_ctx *ctx, const float *X, const float *y, uint32_t n, const float *norm,
                  const float *params, float *grad, float *loss);
/* Predicted normalised log-cost of given feature rows (host in / out). */
int g2_model_predict(g2_ctx *ctx, const float *X, uint64_t n, const float *norm,
                     const float *params, float *out);
/* Model used by G2_SCHED_LEARNED in this context. */
int g2_set_model(g2_ctx *ctx, const float *params, const float *norm);

/* ------------------------------------------------------ host-side helpers */

/* Query planner: preset pattern id (0..27 as PresetPatternType,
 * common/graph.h:25-55) -> plan, following Graph(QUERY) + ReMapVertexId
 * (common/graph.h:127-266), GetConditions (common/graph.h:658-699) and
 * Plan::FindRoot..GenerateStoreStrategy (system/plan.h:51-372). */
int g2_plan_preset(int query_id, g2_plan *out);
/* Same for an arbitrary connected query given as an edge list over 0..k-1. */
int g2_plan_build(uint32_t k, const uint32_t *edges, uint32_t nedges,
                  g2_plan *out);

/* .bin CSR I/O (common/graph.h:360-398 and :539-562).  g2_read_bin allocates
 * *row_ptrs / *cols with malloc; free them with g2_free. */
int g2_read_bin(const char *path, uint64_t **row_ptrs, uint32_t **cols,
                uint64_t *n, uint64_t *m);
int g2_write_bin(const char *path, const uint64_t *row_ptrs,
                 const uint32_t *cols, uint64_t n, uint64_t m);
void g2_free(void *p);
/* SNAP text edge list (Graph::readSnapFile, common/graph.h:268-358): lines that
 * start with a digit hold an edge "u v"; ids are shifted by the smallest; rows
 * symmetric and sorted.  preprocess != 0 applies Graph::Preprocess
 * (common/graph.h:720-804): parallel edges and self loops removed, then vertices
 * without neighbours, the rest renumbered in order; the enumeration needs this
 * form.  Arrays malloc'd (g2_free). */
int g2_read_snap(const char *path, int preprocess, uint64_t **row_ptrs, uint32_t **cols,
                 uint64_t *n, uint64_t *m);

/* .vbmap view-bin partition (view/view_bin_manager.h:34-94): "nbins b0 b1 ...".
 * Writes `n` bin ids; all-zero when nbins == 1. */
int g2_write_vbmap(const char *path, uint32_t nbins, const uint32_t *bins,
                   uint64_t n);
int g2_read_vbmap(const char *path, uint64_t n, uint32_t *nbins,
                  uint32_t *bins);

/*
 * Views (host only).  The view of a root set S is the ball B of radius `radius`
 * around S, ids renumbered 0..|B|-1 in ascending global order (so id
 * comparisons agree with the whole graph); vertices within `row_radius` of S
 * keep their neighbours inside B, the others an empty row.  With G2_VIEW_UPPER
 * the ball of each source s is walked through vertices larger than s only
 * (queries whose conditions place every matched vertex above the root's
 * image: cliques, cycles); with G2_VIEW_FORWARD rows keep only their entries
 * above their own vertex (queries whose conditions order every position above
 * all earlier ones: cliques; every candidate then lies above its parent's
 * image); with G2_VIEW_EGO (radius 1 only) rows keep only the entries (u, y)
 * for which some root s of S has u and y in N[s]: a radius-1 search from s
 * reads nothing outside N[s] (maximal cliques: P, X and their rows; matches:
 * every query vertex is adjacent to the root).  Every embedding rooted in S lies in B and uses only
 * rows of vertices within the query's back-neighbour distance, so a search
 * over the view from S's local ids finds exactly what it finds in the whole
 * graph (view/view_bin.h:40-159 keeps global ids and whole rows instead).
 * Sources of degree < min_root_degree are dropped.  Arrays are malloc'd;
 * release them with g2_view_free.
 */
typedef struct g2_view {
    uint64_t *row_ptrs;     /* n + 1                                          */
    uint32_t *cols;         /* m                                              */
    uint32_t *fwd_offsets;  /* n: neighbours <= v in row v                     */
    uint32_t *sources;      /* nsrc local ids, in the given order             */
    uint32_t *ids;          /* n: global id of each view vertex               */
    uint64_t n, m, nsrc;
    uint32_t max_fwd;       /* max forward degree inside the view             */
} g2_view;
int g2_view_materialize(const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n,
                        const uint32_t *sources, uint64_t nsrc, uint32_t radius,
                        uint32_t row_radius, uint32_t min_root_degree, uint32_t flags,
                        g2_view *out);
void g2_view_free(g2_view *view);
/* The same view built by the GPU of `ctx` (the builder G2_VIEW_DEVICE uses in
 * view runs), copied back into malloc'd arrays (release with g2_view_free):
 * radius 1, row radius 1, no G2_VIEW_EGO (else G2_ERR_UNSUPPORTED).  The
 * context's loaded graph is released.  No counterpart in the reference. */
int g2_view_materialize_device(g2_ctx *ctx, const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n,
                               const uint32_t *sources, uint64_t nsrc, uint32_t min_root_degree,
                               uint32_t flags, g2_view *out);
/* Radius, row radius, root degree and flags (G2_VIEW_UPPER, G2_VIEW_FORWARD) a plan's views
 * need (system/plan.h:51-73 derives the reference's single hop count from the
 * same query distances). */
int g2_plan_view_radius(const g2_plan *plan, uint32_t *radius, uint32_t *row_radius,
                        uint32_t *root_degree, uint32_t *flags);
/* Greedy bins over the roots 0..n-1 in id order: a bin closes when its view
 * would exceed max_bytes (its exact size, counted as the bin grows, up to 48
 * bytes of alignment; a bin holds at least one root).  bin_of: n entries (a
 * .vbmap body).  Host memory: a byte per vertex per planning thread (at most
 * 8 GB); views cost each producer 4 bytes per vertex of the graph. */
int g2_view_bins(const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n, uint32_t radius,
                 uint32_t row_radius, uint32_t min_root_degree, uint32_t flags,
                 uint64_t max_bytes, uint32_t *bin_of, uint32_t *nbins);

/* The reference's kcore bins (kmeans/kcore.cpp:193-228): core[v] of a graph in
 * degeneracy order (ascending, so every shell is a run of ids); each shell is
 * dealt to the nbins bins in consecutive chunks of shell size / nbins + 1. */
int g2_shell_bins(const uint32_t *core, uint64_t n, uint32_t nbins, uint32_t *bin_of);

/* The reference's bin balancing for several devices (view/view_bin_manager.h:
 * 95-184, flags -ds / -dst / -dr): with split_times > 0 the bin whose factor
 * (degree sum of its roots) is furthest above the mean is cut in two until
 * there are (nbins / devices + split_times) * devices bins, its roots dealt
 * alternately in descending degree order; with split_times > 0 or reorder the
 * bins are then numbered by descending factor.  bin_of (n entries,
 * G2_VIEW_NO_BIN for non-roots) is rewritten; *out_nbins receives the count. */
int g2_view_bins_rebalance(const uint64_t *row_ptrs, uint64_t n, uint32_t *bin_of, uint32_t nbins,
                           uint32_t devices, uint32_t split_times, int reorder, uint32_t *out_nbins);

/*
 * Degeneracy order (kmeans/kcore.cpp:103-191): k-core shells in increasing core
 * number, vertices of a shell by increasing degree (ties: lower old id), then
 * recode ids so that u < v means "u earlier in the order".
 * core (optional, n entries) receives core numbers in OLD ids; perm (n entries)
 * receives new_id[old_id].  g2_recode applies a permutation to a CSR
 * (neighbour lists re-sorted); outputs preallocated by the caller.
 */
int g2_degeneracy_order(const uint64_t *row_ptrs, const uint32_t *cols,
                        uint64_t n, uint32_t *perm, uint32_t *core);
int g2_recode(const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n,
              const uint32_t *perm, uint64_t *out_row_ptrs,
              uint32_t *out_cols);

/*
 * Seeded synthetic graphs, written as a symmetric, deduplicated, self-loop free
 * CSR (*row_ptrs / *cols malloc'd; free with g2_free).  Every random draw is a
 * counter-based hash of (seed, stream, index), so any thread count gives the
 * same graph.
 *   er:      G(n, p) plus `nplanted` cliques of size `planted_size` on disjoint
 *            random vertex sets;
 *   rmat:    2^scale vertices, edge_factor * 2^scale generated edges with
 *            quadrant probabilities (a, b, c, 1-a-b-c), plus `nplanted` cliques
 *            of sizes uniform in [planted_min, planted_max];
 *   chunglu: n vertices, expected degree w_i ~ (i+1)^(-1/(gamma-1)) scaled to
 *            avg_degree, n*avg_degree/2 edges drawn proportional to w.
 */
int g2_gen_er(uint64_t n, double p, uint32_t nplanted, uint32_t planted_size,
              uint64_t seed, uint64_t **row_ptrs, uint32_t **cols,
              uint64_t *out_n, uint64_t *out_m);
int g2_gen_rmat(uint32_t scale, uint32_t edge_factor, double a, double b,
                double c, uint32_t nplanted, uint32_t planted_min,
                uint32_t planted_max, uint64_t seed, uint64_t **row_ptrs,
                uint32_t **cols, uint64_t *out_n, uint64_t *out_m);
/* The same seeded R-MAT graph (same rows, planted cliques included) built on
 * the device straight into the context, as if loaded by g2_load_csr; *m_out
 * receives its directed entry count.  For scales whose host build is slow
 * (scale 26, edge factor 28: 3.6 G entries).  scale <= 30.  Test and benchmark
 * input; no counterpart in the reference, which reads graphs from files. */
int g2_gen_rmat_device(g2_ctx *ctx, uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                       uint32_t nplanted, uint32_t planted_min, uint32_t planted_max, uint64_t seed,
                       uint64_t *m_out);
int g2_gen_chunglu(uint64_t n, double gamma, double avg_degree, uint64_t seed,
                   uint64_t **row_ptrs, uint32_t **cols, uint64_t *out_n,
                   uint64_t *out_m);

#ifdef __cplusplus
}
#endif

#endif /* G2_AIMD_H */
