// g2_kernels.h - argument blocks and launchers of the device kernels
// (internal to libg2aimd.so; the public surface is include/g2_aimd.h).
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

#include "g2_aimd.h"

namespace g2 {

// Bits of the device status word.
constexpr int kStatusDeferOverflow = 1;  // deferred-task list full
constexpr int kStatusHistOverflow = 2;   // clique larger than the histogram
constexpr int kStatusStackOverflow = 4;  // GMatch candidate stack exhausted
constexpr int kStatusBadPlan = 8;        // plan arrays inconsistent
constexpr int kStatusWaitLimit = 16;     // a bounded device wait ran out
constexpr int kStatusDeadline = 32;      // the run's time budget ran out (MCE)

// An MCE pass entry with this bit set is a spilled record id, else a task id.
constexpr uint32_t kRecordBit = 0x80000000u;
// Depth word of a record slot whose reservation ran past the buffer's end.
constexpr uint32_t kVoidRecord = 0xffffffffu;

struct MceArgs {
    const uint64_t *rp;
    const uint32_t *ci;
    const uint32_t *fo;             // fo[v]: offset in N(v) of the first neighbour > v
    const uint32_t *tasks;          // root vertex of each task
    const uint32_t *task_index;     // optional: the task ids this pass runs (else 0..ntasks-1)
    const uint32_t *task_part;      // optional per task id: (nparts << 16) | part of a split root
    uint32_t split_depth;           // split roots deal out their depth-split_depth subtrees (>= 1)
    uint64_t *root_cost;            // optional per task id: SM cycles spent on the task
    uint64_t ntasks;                // tasks in this pass (if ntasks_dev is null)
    const unsigned long long *ntasks_dev;  // else: task count read from device memory
    unsigned long long *head;       // device queue head
    uint32_t chunk;                 // tasks grabbed per atomic
    uint32_t hist_len;
    uint32_t *scratch;              // warps * words_per_warp words
    uint64_t words_per_warp;        // multiple of 64
    unsigned long long *out;        // [0] count, [1 + s] hist[s]
    uint32_t *deferred;             // task ids deferred to a larger pass
    unsigned long long *ndeferred;
    uint64_t deferred_cap;
    uint64_t *root_nodes;           // optional, per task id
    uint64_t *root_cliques;         // optional: maximal cliques found per task id
    unsigned long long *hist_dev;   // optional: per-root histogram here (a one-warp pass
                                    // whose slab is the spill slab) instead of the slab's head
    unsigned long long *work;       // optional: work model W in bytes (metrics kernel)
    int *status;
    // handed-off search-tree nodes (record: task, depth, pool offset / 64, nb,
    // then P, X, R rows of rec_words words; rec_stride words each)
    uint32_t *records;
    uint32_t *ready;                // per record slot: epoch of the run that published it
    unsigned long long *nrec;       // records written in this run (append-only)
    uint64_t rec_cap;
    uint32_t rec_stride, rec_words;
    uint32_t *pool;                 // A and B rows of the roots whose tasks spilled
    unsigned long long *npool;      // 64-word units used
    uint64_t pool_cap;              // words
    uint64_t spill_cycles;          // 0: no hand-off in this pass
    unsigned long long *qctl;       // record queue: [kQHead] tickets taken, [kQOut] outstanding work
    uint32_t epoch;                 // ready word of records published in this run (read from epoch_dev)
    const uint32_t *epoch_dev;      // the run's epoch, bumped on the device at the run's start
    uint64_t wait_cycles;           // longest wait of a warp for its ticket's record
    const unsigned long long *deadline;  // optional: %globaltimer (ns) past which roots are
                                         // dropped (set on the device by deadline_set)
};
constexpr int kQHead = 0, kQOut = 1;
constexpr uint32_t kMatchRecordWords = 32;  // stride of a plan-walk record

size_t mce_smem_bytes(int wpl, int warps_per_block);
// Resident CTAs per SM of the kernel a launch with these parameters runs (0 on error).
int mce_blocks_per_sm(int wpl, int warps_per_block, bool metrics);
int match_blocks_per_sm(int wpl, int warps_per_block, bool metrics, int ctas_per_sm, uint32_t p0_words);
cudaError_t mce_launch(int wpl, const MceArgs &a, int blocks, int warps_per_block, cudaStream_t st);
// Advance a run's hand-off epoch in stream order (skipping 0, the value of a
// never-published ready word), so runs captured in a CUDA graph stay distinct
// when the graph is replayed.
cudaError_t epoch_bump(uint32_t *epoch_dev, cudaStream_t st);
// *deadline = the device's %globaltimer now + budget_ns, in stream order.
cudaError_t deadline_set(unsigned long long *deadline, unsigned long long budget_ns, cudaStream_t st);
// In stream order: kStatusDeferOverflow into *status if *left (entries no pass
// walked) is nonzero.
cudaError_t flag_left(const unsigned long long *left, int *status, cudaStream_t st);

// Plan in device-friendly form: everything by POSITION.
struct DevPlan {
    uint32_t k;
    uint32_t bn_count[G2_MAX_QUERY];
    uint32_t bn_pos[G2_MAX_QUERY][G2_MAX_QUERY];       // back neighbours as positions
    uint32_t cond_count[G2_MAX_QUERY];
    uint32_t cond_op[G2_MAX_QUERY][G2_MAX_QUERY];      // condition of position p vs ...
    uint32_t cond_pos[G2_MAX_QUERY][G2_MAX_QUERY];     // ... the vertex matched at this position
    uint32_t share[G2_MAX_QUERY];                      // prefix intersection computed one level early
    uint32_t pre_bn_count[G2_MAX_QUERY];
    uint32_t pre_bn_pos[G2_MAX_QUERY][G2_MAX_QUERY];
    uint32_t pre_cond_count[G2_MAX_QUERY];
    uint32_t pre_cond_op[G2_MAX_QUERY][G2_MAX_QUERY];
    uint32_t pre_cond_pos[G2_MAX_QUERY][G2_MAX_QUERY];
    uint32_t after_bn_count[G2_MAX_QUERY];
    uint32_t after_bn_pos[G2_MAX_QUERY][G2_MAX_QUERY];
    uint32_t after_cond_count[G2_MAX_QUERY];
    uint32_t after_cond_op[G2_MAX_QUERY][G2_MAX_QUERY];
    uint32_t after_cond_pos[G2_MAX_QUERY][G2_MAX_QUERY];
    uint32_t clique;        // 1: every position adjacent to all earlier ones, strictly increasing images
};

struct MatchArgs {
    const uint64_t *rp;
    const uint32_t *ci;
    const uint32_t *fo;
    const uint32_t *tasks;
    const uint32_t *task_index;
    const uint32_t *task_part;      // optional per task: (nparts << 16) | part of a split root
    uint64_t *root_cost;            // optional per task: SM cycles spent on the task
    uint64_t ntasks;
    const unsigned long long *ntasks_dev;  // optional: task count read from device memory
    unsigned long long *head;
    uint32_t chunk;
    uint32_t *scratch;
    uint64_t words_per_warp;
    unsigned long long *out;        // [0] count
    unsigned long long *work;       // optional: work model W in bytes (metrics kernel)
    uint32_t *deferred;
    unsigned long long *ndeferred;
    uint64_t deferred_cap;
    uint64_t *root_nodes;           // optional: embeddings counted per task
    int *status;
    // hand-off of pending plan-walk work to idle warps (g2_handoff.cuh); record:
    // [task, level, kind, ncand, M[0..7], window pos (2), end (2), candidates (16)]
    uint32_t *records;
    uint32_t *ready;
    unsigned long long *nrec;
    uint64_t rec_cap;
    uint32_t rec_stride;
    unsigned long long *qctl;
    uint32_t epoch;                 // ready word of records published in this run (read from epoch_dev)
    const uint32_t *epoch_dev;      // the run's epoch, bumped on the device at the run's start
    uint64_t wait_cycles;
    uint64_t spill_cycles;          // 0: no hand-off
    uint32_t p0_words;              // shared words per warp for P0 (see match_p0_words)
    const unsigned long long *deadline;  // optional: %globaltimer (ns) past which roots are dropped
};

// Shared-memory words per warp the clique path needs besides its row buffer:
// P0 staged for the symmetric-row walk (k > 5 or the metrics build), or the
// P0 filter and hit queue of the lane-parallel counting (k <= 5); none for
// plan walks (non-clique plans).
uint32_t match_p0_words(int wpl, bool clique_path, uint32_t k, bool metrics);
size_t match_smem_bytes(int wpl, int warps_per_block, uint32_t p0_words);
cudaError_t match_launch(const DevPlan &plan, const MatchArgs &a, int blocks, int warps_per_block,
                         cudaStream_t st, bool clique_path, int wpl, int ctas_per_sm);

// Sort each row of `in` (device CSR rows given by rp) into `out`, in calls of at
// most max_chunk entries (kcore.cu); synchronous.
cudaError_t sort_rows_device(const uint64_t *rp, uint64_t n, uint64_t m, const uint32_t *in, uint32_t *out,
                             uint64_t max_chunk, int sms);
// Degeneracy order of a CSR on the device (kcore.cu); synchronous.
cudaError_t degeneracy_order_device(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint32_t *perm,
                                    uint32_t *core, int sms, uint64_t *rounds);
// The CSR with vertex v renamed perm[v], rows sorted (kcore.cu); synchronous.
// new_rp (n+1) and new_ci (m) are allocated here (cudaMalloc); rows are sorted
// in calls of at most max_chunk entries (a row longer than that: NotSupported).
cudaError_t recode_device(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint64_t m, const uint32_t *perm,
                          uint64_t max_chunk, int sms, uint64_t **new_rp, uint32_t **new_ci);

// Learned root-cost model (costmodel.cu).
size_t model_smem_bytes();
cudaError_t features_launch(const uint64_t *rp, const uint32_t *ci, const uint32_t *fo, const uint32_t *core,
                            const uint32_t *src, uint64_t n, float *out, int sms, cudaStream_t st);
cudaError_t train_step_launch(const float *X, const float *Y, const uint32_t *idx, uint32_t n, const float *params,
                              const float *norm, float *grad, float *loss, cudaStream_t st);
cudaError_t adam_launch(float *params, float *mom, float *vel, const float *grad, float lr, int step,
                        cudaStream_t st);
cudaError_t score_launch(const uint64_t *rp, const uint32_t *ci, const uint32_t *fo, const uint32_t *core,
                         const uint32_t *src, uint64_t n, const float *X, const float *params, const float *norm,
                         float *pred, float *cost, float *total, int sms, cudaStream_t st);

}  // namespace g2
