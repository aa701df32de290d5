// mce.cu - maximal clique enumeration (Bron-Kerbosch, Tomita pivot) for sm_100a.
//
// Replaces app_BK's BFS over labelled records (app_BK/BK.h:323-474 driven by
// system/pipeline_executor.h:151-207) with a persistent kernel: each warp pulls
// root tasks from a device atomic queue and walks the root's search tree depth
// first, with its DFS frames in an HBM scratch slab.
//
// Per root v (ids in degeneracy order, so |P0| <= degeneracy):
//   P0 = N(v) ∩ (v, ∞)  (p vertices, local index 0..p-1, W = ceil(p/32) words)
//   X0 = N(v) ∩ [0, v)
//   A[i]  = N(P0[i]) ∩ P0          as a p-bit row          (p x W words)
//   B[j]  = N(x_j) ∩ P0 for x_j ∈ X0, rows that are all zero dropped
// A search-tree node is (R, P ⊆ P0, X = X_P0 ⊆ P0 plus a list of B rows).
// Child for q: P' = P ∩ A[q], X_P0' = X_P0 ∩ A[q], list' = {x in list : bit q
// of B[x]}; then q moves from P to X (sequential BK, app_BK/BK.h:226,278).
// Pivot: argmax |P ∩ row(u)| over u ∈ P ∪ X, ties to the larger vertex id
// (app_BK/BK.h:314; X0 ids < v < P0 ids and both are kept sorted), so the tree
// is exactly the reference's and per-root node counts match the oracle.
//
// Hand-off (load balance inside a root): every spill_cycles SM cycles a walk
// checks whether idle warps hold tickets beyond the published records
// (g2_handoff.cuh); if so it writes the pending branches of its shallowest open
// level as records (node depth, P, X and the path R as P0 bitmaps; at its own
// level it keeps the first branch) and keeps walking.  A root's rows go once to
// a shared row pool.  Idle warps run the records, each rebuilding its B list as
// the root's kept rows that contain R.  Every node is still visited exactly
// once, in the same tree, so counts, histograms and per-root node counts do not
// change.  Search trees of the dense cores of power-law graphs are chains at the
// top (one branch per node for many levels), which is why the split is taken
// where the walk is, not at a fixed depth.
//
// A root whose rows or frames do not fit in the warp's slab (or whose p needs
// more than 32*WPL words) is deferred whole, before anything is written or
// counted: the host re-runs deferred entries with a larger slab per warp (fewer
// warps), then with one warp owning the whole scratch, then (synchronous runs)
// on a managed spill slab.  An entry that has handed work off is never deferred:
// on slab overflow it hands off everything instead.  The only waits are the
// bounded ones of the record queue.
#include <cstdint>

#include "g2_bitrows.cuh"
#include "g2_device.cuh"
#include "g2_handoff.cuh"
#include "g2_kernels.h"

namespace g2 {

namespace {


// slab frame per open level: P, X, Qr rows, list offset, list length, branch taken
__device__ __forceinline__ uint32_t frame_words(uint32_t W) { return 3u * W + 3u; }

__device__ void defer_entry(const MceArgs &a, uint32_t entry) {
    if (lane_id() == 0) {
        unsigned long long d = atomicAdd(a.ndeferred, 1ull);
        if (d < a.deferred_cap) a.deferred[d] = entry;
        else atomicOr(a.status, kStatusDeferOverflow);
    }
}

// Sum of degrees of the P0 vertices whose bits are set in a distributed row.
template <int WPL>
__device__ __forceinline__ unsigned long long row_degree_sum(const Row<WPL> &r, const uint64_t *rp,
                                                             const uint32_t *ci, uint64_t split) {
    const uint32_t lane = lane_id();
    unsigned long long s = 0;
#pragma unroll
    for (int k = 0; k < WPL; k++) {
        uint32_t word = r.w[k];
        while (word) {
            uint32_t b = __ffs(word) - 1;
            word &= word - 1;
            uint32_t u = ldg(ci + split + (lane + 32u * k) * 32u + b);
            s += ldg(rp + u + 1) - ldg(rp + u);
        }
    }
    return warp_sum_u64(s);
}

template <int WPL>
__device__ __forceinline__ uint32_t row_popc(const Row<WPL> &r) {
    uint32_t c = 0;
#pragma unroll
    for (int k = 0; k < WPL; k++) c += __popc(r.w[k]);
    return (uint32_t)warp_sum_u64(c);
}

// Lowest set bit of a distributed row (all lanes), ~0u if the row is empty.
template <int WPL>
__device__ __forceinline__ uint32_t row_lowest(const Row<WPL> &r) {
    const uint32_t lane = lane_id();
    uint32_t key = 0xffffffffu;
#pragma unroll
    for (int s = WPL - 1; s >= 0; s--)
        if (r.w[s]) key = 32u * (uint32_t)s + lane;  // word index lane + 32*s
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        uint32_t y = __shfl_xor_sync(G2_FULL, key, o);
        key = y < key ? y : key;
    }
    if (key == 0xffffffffu) return key;
    return key * 32u + (uint32_t)(__ffs(row_word(r, key)) - 1);
}

template <int WPL>
__device__ __forceinline__ void row_assign_bit(Row<WPL> &r, uint32_t q, bool on) {
    const uint32_t lane = lane_id(), qw = q >> 5, bit = 1u << (q & 31u);
#pragma unroll
    for (int s = 0; s < WPL; s++)
        if (lane + 32u * s == qw) r.w[s] = on ? (r.w[s] | bit) : (r.w[s] & ~bit);
}

template <int WPL>
__device__ __forceinline__ void row_load_cg(Row<WPL> &r, const uint32_t *src, uint32_t W) {
    const uint32_t lane = lane_id();
#pragma unroll
    for (int s = 0; s < WPL; s++) {
        uint32_t w = lane + 32u * s;
        r.w[s] = w < W ? __ldcg(src + w) : 0u;
    }
}

// The rows a walk reads: slab rows of a root task, or pool rows of a record.
struct Rows {
    const uint32_t *A;   // p rows of W words
    const uint32_t *B;   // nb kept X0 rows of W words
    const uint32_t *xv;  // metrics: X0 vertex of each kept row
    uint64_t pool_off;   // offset of the rows in the pool, ~0 while they live in the slab
};

// Record layout: [task, depth, pool offset / 64, nb, P (W), X (W), R (W)]; the
// ready word of slot i is ready[i] (a separate array that holds nothing but
// epochs, whatever the record stride of earlier runs was).
constexpr uint32_t kRecRows = 4;

// Rows of a root task go to the pool before its first records reference them.
template <bool METRICS>
__device__ bool ensure_pooled(const MceArgs &a, uint32_t p, uint32_t nb, uint32_t W, Rows &rows) {
    const uint32_t lane = lane_id();
    if (rows.pool_off != ~0ull) return true;
    const uint64_t words = (uint64_t)(p + nb) * W + (METRICS ? nb : 0u);
    const uint64_t units = (words + 63u) >> 6;
    unsigned long long off = 0;
    if (lane == 0) off = atomicAdd(a.npool, (unsigned long long)units);
    off = __shfl_sync(G2_FULL, off, 0);
    if ((off + units) << 6 > a.pool_cap) return false;
    uint32_t *dst = a.pool + (off << 6);
    for (uint64_t i = lane; i < (uint64_t)p * W; i += 32) dst[i] = rows.A[i];
    for (uint64_t i = lane; i < (uint64_t)nb * W; i += 32) dst[(uint64_t)p * W + i] = rows.B[i];
    if (METRICS)
        for (uint32_t i = lane; i < nb; i += 32) dst[(uint64_t)(p + nb) * W + i] = rows.xv[i];
    __syncwarp();
    rows.pool_off = off << 6;
    rows.A = dst;
    rows.B = dst + (uint64_t)p * W;
    rows.xv = dst + (uint64_t)(p + nb) * W;
    return true;
}

// Write records k, k+1, ... for the branches Q of one level (ascending; each
// branch's P and X see the earlier ones moved from P to X, sequential BK).
// R is the level's path; depth the children's depth.  Returns the next slot.
template <int WPL>
__device__ unsigned long long emit_level(const MceArgs &a, unsigned long long k, uint32_t task, uint32_t depth,
                                         Row<WPL> Pl, Row<WPL> Xl, Row<WPL> Ql, const Row<WPL> &R,
                                         const Rows &rows, uint32_t nb, uint32_t W) {
    const uint32_t lane = lane_id();
    for (;;) {
        const uint32_t q = row_lowest(Ql);
        if (q == 0xffffffffu) break;
        row_assign_bit(Ql, q, false);
        Row<WPL> aq, cp, cx, cr;
        row_load(aq, rows.A + (uint64_t)q * W, W);
#pragma unroll
        for (int s = 0; s < WPL; s++) {
            cp.w[s] = Pl.w[s] & aq.w[s];
            cx.w[s] = Xl.w[s] & aq.w[s];
            cr.w[s] = R.w[s];
        }
        row_assign_bit(cr, q, true);
        uint32_t *rec = a.records + k * a.rec_stride;
        k++;
        if (lane == 0) {
            rec[0] = task;
            rec[1] = depth;
            rec[2] = (uint32_t)(rows.pool_off >> 6);
            rec[3] = nb;
        }
        row_store(cp, rec + kRecRows, W);
        row_store(cx, rec + kRecRows + W, W);
        row_store(cr, rec + kRecRows + 2u * W, W);
        row_assign_bit(Pl, q, false);
        row_assign_bit(Xl, q, true);
    }
    return k;
}

// Pending-branch count of every frame level below d, as (first level with any, its count).
template <int WPL>
__device__ void shallowest_pending(const uint32_t *frames, uint32_t d, uint32_t W, uint32_t *level,
                                   uint32_t *count) {
    const uint32_t lane = lane_id(), FR = frame_words(W);
    *level = d;
    *count = 0;
    for (uint32_t l = 0; l < d; l++) {
        uint32_t c = 0;
        for (uint32_t w = lane; w < W; w += 32) c += __popc(frames[(uint64_t)l * FR + 2u * W + w]);
        c = (uint32_t)warp_sum_u64(c);
        if (c) {
            *level = l;
            *count = c;
            return;
        }
    }
}

// Path R of frame level l: the entry node's R plus the branches taken at levels < l.
template <int WPL>
__device__ Row<WPL> path_of(const uint32_t *frames, uint32_t l, uint32_t W, const Row<WPL> &Rbase) {
    const uint32_t FR = frame_words(W);
    Row<WPL> R = Rbase;
    for (uint32_t j = 0; j < l; j++) row_assign_bit(R, frames[(uint64_t)j * FR + 3u * W + 2u], true);
    return R;
}

// Hand the pending branches of the shallowest open level (its subtrees are the
// largest) to idle warps and keep walking.  At the current level d the first
// branch stays with this warp.  Returns false if nothing was handed off.
template <int WPL, bool METRICS>
__device__ __noinline__ bool donate(const MceArgs &a, uint32_t task, uint32_t d0, uint32_t d, const Row<WPL> &P,
                                    const Row<WPL> &X, Row<WPL> &Qr, const Row<WPL> &Rbase, uint32_t *frames,
                                    uint32_t W, uint32_t p, uint32_t nb, Rows &rows, bool *full) {
    const uint32_t FR = frame_words(W);
    uint32_t l, cnt;
    shallowest_pending<WPL>(frames, d, W, &l, &cnt);
    uint32_t q0 = 0xffffffffu;
    if (cnt == 0) {  // only the current level: keep its first branch
        q0 = row_lowest(Qr);
        cnt = row_popc(Qr);
        cnt = cnt ? cnt - 1 : 0;
        if (cnt == 0) return false;
    }
    if (!ensure_pooled<METRICS>(a, p, nb, W, rows)) {
        *full = true;
        return false;
    }
    const unsigned long long k0 = reserve_records(a, cnt);
    if (k0 == ~0ull) {
        *full = true;
        return false;
    }
    const Row<WPL> R = path_of<WPL>(frames, l, W, Rbase);
    Row<WPL> Pl, Xl, Ql;
    uint32_t *f = frames + (uint64_t)l * FR;
    if (l < d) {
        row_load(Pl, f, W);
        row_load(Xl, f + W, W);
        row_load(Ql, f + 2u * W, W);
    } else {
        Pl = P;
        Xl = X;
        Ql = Qr;
        row_assign_bit(Pl, q0, false);  // q0 runs first here, so later siblings see it in X
        row_assign_bit(Xl, q0, true);
        row_assign_bit(Ql, q0, false);
    }
    const unsigned long long k1 = emit_level<WPL>(a, k0, task, d0 + l + 1u, Pl, Xl, Ql, R, rows, nb, W);
    publish_records(a, k0, k1);
    if (l < d) {
        Row<WPL> z;
        row_zero(z);
        row_store(z, f + 2u * W, W);  // the donated branches leave the frame
        __syncwarp();
    } else {
        row_zero(Qr);
        row_assign_bit(Qr, q0, true);
    }
    return true;
}

// Hand every pending branch of levels 0..d to records (level d is the register
// state P, X, Qr) and end the walk.  Returns false, with nothing published
// that a claimer would run, if the buffers are full.
template <int WPL, bool METRICS>
__device__ __noinline__ bool spill_all(const MceArgs &a, uint32_t task, uint32_t d0, uint32_t d, const Row<WPL> &P,
                                       const Row<WPL> &X, const Row<WPL> &Qr, const Row<WPL> &Rbase,
                                       const uint32_t *frames, uint32_t W, uint32_t p, uint32_t nb, Rows &rows) {
    const uint32_t lane = lane_id(), FR = frame_words(W);
    uint32_t need = row_popc(Qr);
    for (uint32_t l = 0; l < d; l++) {
        uint32_t c = 0;
        for (uint32_t w = lane; w < W; w += 32) c += __popc(frames[(uint64_t)l * FR + 2u * W + w]);
        need += (uint32_t)warp_sum_u64(c);
    }
    if (need == 0) return true;  // nothing pending: the walk is complete
    if (!ensure_pooled<METRICS>(a, p, nb, W, rows)) return false;
    const unsigned long long k0 = reserve_records(a, need);
    if (k0 == ~0ull) return false;
    unsigned long long k = k0;
    Row<WPL> R = Rbase;
    for (uint32_t l = 0; l <= d; l++) {
        const uint32_t *f = frames + (uint64_t)l * FR;
        if (l < d) {
            Row<WPL> Pl, Xl, Ql;
            row_load(Pl, f, W);
            row_load(Xl, f + W, W);
            row_load(Ql, f + 2u * W, W);
            k = emit_level<WPL>(a, k, task, d0 + l + 1u, Pl, Xl, Ql, R, rows, nb, W);
            row_assign_bit(R, f[3u * W + 2u], true);
        } else {
            k = emit_level<WPL>(a, k, task, d0 + l + 1u, P, X, Qr, R, rows, nb, W);
        }
    }
    publish_records(a, k0, k);
    return true;
}

enum : int { kTaskDone = 0, kTaskDeferred = 1 };

// Has the run's time budget (MceArgs::deadline, %globaltimer ns) run out?
// Warp-uniform.
__device__ __forceinline__ bool deadline_passed(const MceArgs &a) {
    if (!a.deadline) return false;
    unsigned long long now = 0;
    if (lane_id() == 0) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    now = __shfl_sync(G2_FULL, now, 0);
    return now > *a.deadline;
}

// Run one entry: a root task (entry < 2^31) or a handed-off record (entry has
// kRecordBit set).  With METRICS the work model W (in 4-byte words) of the
// reference's tree is accumulated: per node with P ∪ X non-empty,
// sum_{u in P∪X} (|P| + deg u) for pivot scoring plus
// sum_{q in P \ N(pivot)} (|P ∪ X| + deg q) for the children.
template <int WPL, bool METRICS, bool BUDGET>
__device__ int mce_task(const MceArgs &a, uint32_t entry, uint32_t *S, uint32_t *cand, uint32_t *rowbuf,
                        long long c0, uint32_t *task_out) {
    const uint32_t lane = lane_id();
    const uint64_t *rp = a.rp;
    const uint32_t *ci = a.ci;
    const bool is_rec = (entry & kRecordBit) != 0;
    const uint32_t *rec = is_rec ? a.records + (uint64_t)(entry & ~kRecordBit) * a.rec_stride : nullptr;
    // record words are read past L1 (two records share a cache line, and a line
    // another warp of this SM read earlier may predate this record)
    if (is_rec && __ldcg(rec + 1) == kVoidRecord) {  // slot of a reservation that did not fit
        *task_out = ~0u;
        return kTaskDone;
    }
    const uint32_t task = is_rec ? __ldcg(rec) : entry;
    const uint32_t d0 = is_rec ? __ldcg(rec + 1) : 0u;  // depth of the entry node (R has d0 + 1 vertices)
    *task_out = task;
    const uint32_t v = a.tasks[task];
    const uint64_t lo = ldg(rp + v), hi = ldg(rp + v + 1);
    // static heavy-root split: every part walks the nodes above depth D (they are
    // the same in every part; part 0 counts them) and owns the depth-D subtrees
    // whose ordinal, in depth-first order, is congruent to part mod nparts
    const uint32_t tp = (a.task_part && !is_rec) ? a.task_part[task] : (1u << 16);
    const uint32_t nparts = tp >> 16, part = tp & 0xffffu;
    const uint32_t D = nparts > 1 ? (a.split_depth ? a.split_depth : 1u) : 0u;
    if (!is_rec && (lo == hi || (part != 0 && ldg(a.fo + v) == hi - lo))) {  // no neighbours (app_BK/BK.h:335-336) or P empty
        return kTaskDone;
    }
    uint32_t branch = 0;  // ordinal of the next depth-D subtree
    const uint64_t split = lo + ldg(a.fo + v);
    const uint32_t p = (uint32_t)(hi - split);
    const uint32_t nx = (uint32_t)(split - lo);
    if (p == 0) {  // P empty, X non-empty: one record, not maximal
        if (METRICS) {  // its pivot scan still reads every X0 list
            unsigned long long sx = 0;
            for (uint32_t li = lane; li < nx; li += 32) {
                const uint32_t u = ldg(ci + lo + li);
                sx += ldg(rp + u + 1) - ldg(rp + u);
            }
            sx = warp_sum_u64(sx);
            if (lane == 0) atomicAdd(a.work, sx * 4ull);
        }
        if (a.root_nodes && lane == 0) atomicAdd(reinterpret_cast<unsigned long long *>(a.root_nodes + task), 1ull);
        return kTaskDone;
    }
    const uint32_t W = (p + 31u) >> 5;
    if (W > 32u * WPL) return kTaskDeferred;
    const uint64_t SW = a.words_per_warp;
    const uint32_t FR = frame_words(W);
    const uint64_t fr0 = SW >= (uint64_t)(p + 1) * FR ? SW - (uint64_t)(p + 1) * FR : 0;
    unsigned long long *hist_local = a.hist_dev ? a.hist_dev : reinterpret_cast<unsigned long long *>(S);
    const uint64_t a0 = 2ull * (p + 2);  // after the histogram
    // nothing is written before the slab is known to hold the histogram and frames
    // (a small slab's neighbours are other warps' slabs)
    if (fr0 < a0 + 64) return kTaskDeferred;
    for (uint32_t s = lane; s < p + 2; s += 32) hist_local[s] = 0ull;
    Rows rows;
    uint32_t nb;
    uint64_t l0;  // list region
    Row<WPL> P, X, Qr, Rb;
    uint32_t xlen;
    if (!is_rec) {
        // slab: [hist u64 (p+2)] [A p*W] [xv nx (metrics)] [B nb*W] [lists ...] ... [frames (p+1)*FR]
        const uint64_t xv0 = a0 + (uint64_t)p * W;
        const uint64_t b0 = xv0 + (METRICS ? nx : 0);
        if (fr0 < b0 + 64) return kTaskDeferred;
        // stage P0 in shared memory, then the rows
        for (uint32_t i = lane; i < p; i += 32) cand[i] = ldg(ci + split + i);
        __syncwarp();
        build_forward_rows(rp, ci, a.fo, cand, p, W, S + a0, rowbuf);
        // kept B rows plus their root-list entries must stay below the frames
        const uint64_t cap64 = (fr0 - b0 - 64) / (W + 1);
        const uint32_t cap = cap64 > 0xfffffff0ull ? 0xfffffff0u : (uint32_t)cap64;
        nb = build_back_rows(rp, ci, a.fo, v, lo, nx, cand, p, W, S + b0, METRICS ? S + xv0 : nullptr, cap, rowbuf);
        if (nb == ~0u) return kTaskDeferred;
        __syncwarp();
        rows.A = S + a0;
        rows.B = S + b0;
        rows.xv = S + xv0;
        rows.pool_off = ~0ull;
        // root list: identity over the nb kept rows
        l0 = b0 + (uint64_t)nb * W;
        for (uint32_t i = lane; i < nb; i += 32) S[l0 + i] = i;
        xlen = nb;
#pragma unroll
        for (int s = 0; s < WPL; s++) {
            uint32_t w = lane + 32u * s;
            P.w[s] = w < W ? (w + 1 < W || (p & 31u) == 0 ? G2_FULL : ((1u << (p & 31u)) - 1u)) : 0u;
            X.w[s] = 0u;
            Rb.w[s] = 0u;
        }
    } else {
        // slab: [hist u64 (p+2)] [lists ...] ... [frames]; rows in the pool
        nb = __ldcg(rec + 3);
        rows.pool_off = (uint64_t)__ldcg(rec + 2) << 6;
        rows.A = a.pool + rows.pool_off;
        rows.B = rows.A + (uint64_t)p * W;
        rows.xv = rows.B + (uint64_t)nb * W;
        l0 = a0;
        if (fr0 < l0 + nb + 64) return kTaskDeferred;
        row_load_cg(P, rec + kRecRows, W);
        row_load_cg(X, rec + kRecRows + W, W);
        row_load_cg(Rb, rec + kRecRows + 2u * W, W);
        // the entry node's B list: kept rows adjacent to every vertex of R \ {v}
        xlen = 0;
        for (uint32_t c = 0; c < nb; c += 32) {
            const uint32_t i = c + lane;
            bool ok = i < nb;
            for (uint32_t w = 0; w < W; w++) {
                const uint32_t rw = row_word(Rb, w);
                if (ok && (rows.B[(uint64_t)i * W + w] & rw) != rw) ok = false;
            }
            uint32_t tot;
            const uint32_t pos = warp_scan(ok, tot);
            if (ok) S[l0 + xlen + pos] = i;
            xlen += tot;
        }
    }
#pragma unroll
    for (int s = 0; s < WPL; s++) Qr.w[s] = 0u;
    __syncwarp();
    const uint32_t *Bfull = rows.B;

    // ---- depth-first walk
    uint64_t xoff = l0;
    uint32_t d = 0;  // depth below the entry node
    unsigned long long nodes = 0, cliques = 0, work = 0;
    bool enter = true;
    bool overflow = false, spilled = false, expired = false;
    bool donated = false;  // some branches went to records: the entry can no longer be re-run
    bool may_spill = a.spill_cycles != 0 && nparts == 1 && W <= a.rec_words;
    long long next_check = (long long)a.spill_cycles;
    for (;;) {
        bool want_pop = false;
        if (enter) {
            enter = false;
            if (BUDGET && (nodes & 255u) == 0 && deadline_passed(a)) {  // time budget: drop the root
                expired = true;
                break;
            }
            const bool own = d >= D || part == 0;  // this part counts the node
            const bool at_root = !is_rec && d == 0;
            if (own) nodes++;
            uint32_t anyp = 0, anyx = 0;
#pragma unroll
            for (int s = 0; s < WPL; s++) anyp |= P.w[s], anyx |= X.w[s];
            const bool hp = __any_sync(G2_FULL, anyp != 0);
            const bool hx = __any_sync(G2_FULL, anyx != 0) || xlen > 0;
            unsigned long long npx = 0;  // |P| + |X| (metrics)
            if (METRICS && (hp || hx) && own) {
                // the reference's root record keeps every X0 vertex, also those
                // with no neighbour in P0 that the B list drops (they fall out of
                // every child), so the root node counts all of X0
                const uint32_t np = row_popc(P);
                npx = np + row_popc(X) + (at_root ? nx : xlen);
                unsigned long long sd = row_degree_sum(P, rp, ci, split) + row_degree_sum(X, rp, ci, split);
                unsigned long long sx = 0;
                if (at_root) {
                    for (uint32_t li = lane; li < nx; li += 32) {
                        const uint32_t u = ldg(ci + lo + li);
                        sx += ldg(rp + u + 1) - ldg(rp + u);
                    }
                } else {
                    for (uint32_t li = lane; li < xlen; li += 32) {
                        const uint32_t u = rows.xv[S[xoff + li]];
                        sx += ldg(rp + u + 1) - ldg(rp + u);
                    }
                }
                work += npx * np + sd + warp_sum_u64(sx);
            }
            if (!hp) {
                if (!hx && own) {  // no P and no X: maximal (app_BK/BK.h:78-91)
                    cliques++;
                    if (lane == 0) hist_local[d0 + d + 1]++;
                }
                want_pop = true;
            } else {
                // ---- pivot: max (|P ∩ row|, rank) over P ∪ X_P0 and the B list
                unsigned long long best = 0;
                uint32_t ncand = 0;
#pragma unroll
                for (int s = 0; s < WPL; s++) {
                    uint32_t word = P.w[s] | X.w[s];
                    const uint32_t cnt = __popc(word);
                    uint32_t inc = cnt;
#pragma unroll
                    for (int o = 1; o < 32; o <<= 1) {
                        uint32_t y = __shfl_up_sync(G2_FULL, inc, o);
                        if (lane >= (uint32_t)o) inc += y;
                    }
                    const uint32_t tot = __shfl_sync(G2_FULL, inc, 31);
                    uint32_t pos = ncand + inc - cnt;
                    const uint32_t base = (lane + 32u * s) * 32u;
                    while (word) {
                        uint32_t b = __ffs(word) - 1;
                        word &= word - 1;
                        cand[pos++] = base + b;
                    }
                    ncand += tot;
                }
                __syncwarp();
                for (uint32_t c = 0; c < ncand; c += 32) {
                    const uint32_t k = c + lane;
                    const bool valid = k < ncand;
                    const uint32_t idx = valid ? cand[k] : 0u;
                    const uint32_t *r = rows.A + (uint64_t)idx * W;
                    uint32_t sc = 0;
                    for (uint32_t w = 0; w < W; w++) {
                        const uint32_t pw = row_word(P, w);
                        if (valid) sc += __popc(pw & r[w]);
                    }
                    if (valid) {
                        unsigned long long key = ((unsigned long long)sc << 32) | (unsigned long long)(nb + idx);
                        best = key > best ? key : best;
                    }
                }
                __syncwarp();
                for (uint32_t c = 0; c < xlen; c += 32) {
                    const uint32_t li = c + lane;
                    const bool valid = li < xlen;
                    const uint32_t bi = valid ? S[xoff + li] : 0u;
                    const uint32_t *r = Bfull + (uint64_t)bi * W;
                    uint32_t sc = 0;
                    for (uint32_t w = 0; w < W; w++) {
                        const uint32_t pw = row_word(P, w);
                        if (valid) sc += __popc(pw & r[w]);
                    }
                    if (valid) {
                        unsigned long long key = ((unsigned long long)sc << 32) | (unsigned long long)bi;
                        best = key > best ? key : best;
                    }
                }
                best = warp_max_u64(best);
                const uint32_t rank = (uint32_t)(best & 0xffffffffull);
                const uint32_t *prow =
                    rank >= nb ? rows.A + (uint64_t)(rank - nb) * W : Bfull + (uint64_t)rank * W;
                Row<WPL> pr;
                row_load(pr, prow, W);
#pragma unroll
                for (int s = 0; s < WPL; s++) Qr.w[s] = P.w[s] & ~pr.w[s];
                if (METRICS && own) work += npx * row_popc(Qr) + row_degree_sum(Qr, rp, ci, split);
                // ---- every spill_cycles: hand work to idle warps while they
                // outnumber the records waiting to be claimed
                if (may_spill) {
                    long long el = 0;
                    if (lane == 0) el = clock64() - c0;
                    el = __shfl_sync(G2_FULL, el, 0);
                    if (el > next_check) {
                        if (handoff_wanted(a)) {  // idle warps hold tickets past the last record
                            bool full = false;
                            if (donate<WPL, METRICS>(a, task, d0, d, P, X, Qr, Rb, S + fr0, W, p, nb, rows, &full))
                                donated = true;
                            if (full) may_spill = false;  // buffers full: finish the walk here
                        }
                        next_check = el + (long long)a.spill_cycles;
                    }
                }
            }
        }
        if (!want_pop) {
            // ---- next branch q of the current node: lowest set bit of Qr
            const uint32_t q = row_lowest(Qr);
            if (q == 0xffffffffu) {
                want_pop = true;
            } else {
                const uint32_t qw = q >> 5;
                // q moves from P to X and is consumed from Q
                row_assign_bit(P, q, false);
                row_assign_bit(X, q, true);
                row_assign_bit(Qr, q, false);
                if (d + 1 == D && (branch++ % nparts) != part) continue;  // another part's subtree
                const uint64_t coff = xoff + xlen;
                if (coff + xlen > fr0) {         // child list would reach the frames
                    if (may_spill || donated) {  // hand this level and the ones below to records
                        Row<WPL> P1 = P, X1 = X, Q1 = Qr;
                        row_assign_bit(P1, q, true);
                        row_assign_bit(X1, q, false);
                        row_assign_bit(Q1, q, true);
                        if (spill_all<WPL, METRICS>(a, task, d0, d, P1, X1, Q1, Rb, S + fr0, W, p, nb, rows)) {
                            spilled = true;
                            break;
                        }
                    }
                    overflow = true;
                    break;
                }
                // save the parent state in frame d
                uint32_t *f = S + fr0 + (uint64_t)d * FR;
                row_store(P, f, W);
                row_store(X, f + W, W);
                row_store(Qr, f + 2 * W, W);
                if (lane == 0) {
                    f[3 * W] = (uint32_t)(xoff - l0);
                    f[3 * W + 1] = xlen;
                    f[3 * W + 2] = q;
                }
                // child: P ∩ A[q], X_P0 ∩ A[q], B entries adjacent to q
                Row<WPL> aq;
                row_load(aq, rows.A + (uint64_t)q * W, W);
#pragma unroll
                for (int s = 0; s < WPL; s++) {
                    P.w[s] &= aq.w[s];
                    X.w[s] &= aq.w[s];
                }
                uint32_t clen = 0;
                for (uint32_t c = 0; c < xlen; c += 32) {
                    const uint32_t li = c + lane;
                    const uint32_t bi = li < xlen ? S[xoff + li] : 0u;
                    const bool keep = li < xlen && ((Bfull[(uint64_t)bi * W + qw] >> (q & 31u)) & 1u);
                    uint32_t tot;
                    const uint32_t pos = warp_scan(keep, tot);
                    if (keep) S[coff + clen + pos] = bi;
                    clen += tot;
                }
                __syncwarp();
                xoff = coff;
                xlen = clen;
                d++;
                enter = true;
                continue;
            }
        }
        // ---- pop
        if (d == 0) break;
        d--;
        {
            const uint32_t *f = S + fr0 + (uint64_t)d * FR;
            row_load(P, f, W);
            row_load(X, f + W, W);
            row_load(Qr, f + 2 * W, W);
            xoff = l0 + f[3 * W];
            xlen = f[3 * W + 1];
        }
        __syncwarp();
    }
    if (BUDGET && expired) {  // nothing of this entry is committed (budgeted runs never hand off)
        if (lane == 0) atomicOr(a.status, kStatusDeadline);
        __syncwarp();
        return kTaskDone;
    }
    if (overflow && !spilled) {
        if (!donated) return kTaskDeferred;  // re-run from scratch by a pass with a bigger slab
        if (lane == 0) atomicOr(a.status, kStatusDeferOverflow);  // record buffers full: incomplete
    }
    // ---- commit this entry's results
    __syncwarp();
    if (lane == 0) {
        atomicAdd(a.out, cliques);
        if (a.root_nodes) atomicAdd(reinterpret_cast<unsigned long long *>(a.root_nodes + task), nodes);
        if (a.root_cliques && cliques)
            atomicAdd(reinterpret_cast<unsigned long long *>(a.root_cliques + task), cliques);
        if (METRICS) atomicAdd(a.work, work * 4ull);
    }
    for (uint32_t s = lane; s < p + 2; s += 32) {
        unsigned long long h = hist_local[s];
        if (h) {
            if (s < a.hist_len) atomicAdd(a.out + 1 + s, h);
            else if (a.hist_len) atomicOr(a.status, kStatusHistOverflow);  // hist_len 0: no histogram
        }
    }
    __syncwarp();
    return kTaskDone;
}

template <int WPL, bool METRICS, bool BUDGET>
__device__ __forceinline__ void run_entry(const MceArgs &a, uint32_t entry, uint32_t *S, uint32_t *cand,
                                          uint32_t *rowbuf) {
    long long c0 = 0;
    if (lane_id() == 0) c0 = clock64();
    c0 = __shfl_sync(G2_FULL, c0, 0);
    uint32_t task = 0;
    if (mce_task<WPL, METRICS, BUDGET>(a, entry, S, cand, rowbuf, c0, &task) == kTaskDeferred)
        defer_entry(a, entry);
    else if (a.root_cost && lane_id() == 0 && task != ~0u)
        atomicAdd(reinterpret_cast<unsigned long long *>(a.root_cost + task), (unsigned long long)(clock64() - c0));
}

// Persistent pass.  Phase 1: entries from the task queue (or a deferred list).
// Phase 2 (passes that hand off work): records through the ticket queue of
// g2_handoff.cuh until no work is outstanding.
// BUDGET: the build for runs with a time budget (MceArgs::deadline set); the
// others carry no deadline check.
template <int WPL, bool METRICS, bool BUDGET>
__global__ void __launch_bounds__(256, 3) mce_kernel(MceArgs a) {
    extern __shared__ uint32_t smem[];
    if (a.epoch_dev) a.epoch = *a.epoch_dev;
    const uint32_t wib = threadIdx.x >> 5;
    uint32_t *cand = smem + wib * (32u * 32u * WPL + 32u * WPL);
    uint32_t *rowbuf = cand + 32u * 32u * WPL;
    const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t *S = a.scratch + gw * a.words_per_warp;
    const bool handoff = a.spill_cycles != 0;
    unsigned long long n = a.ntasks;
    if (a.ntasks_dev) {
        n = *a.ntasks_dev;
        if (n > a.deferred_cap) n = a.deferred_cap;
    }
    for (;;) {
        outstanding_add(a, handoff, 1);
        const unsigned long long t0 = grab(a.head, a.chunk);
        if (t0 >= n) {
            outstanding_add(a, handoff, -1);
            break;
        }
        const unsigned long long t1 = t0 + a.chunk < n ? t0 + a.chunk : n;
        for (unsigned long long t = t0; t < t1; t++) {
            if (BUDGET && deadline_passed(a)) {  // time budget spent: start no new root
                if (lane_id() == 0) atomicOr(a.status, kStatusDeadline);
                continue;
            }
            run_entry<WPL, METRICS, BUDGET>(a, a.task_index ? a.task_index[t] : (uint32_t)t, S, cand, rowbuf);
        }
        outstanding_add(a, handoff, -1);
    }
    if (handoff)
        run_record_queue(a, [&](unsigned long long h) {
            run_entry<WPL, METRICS, BUDGET>(a, kRecordBit | (uint32_t)h, S, cand, rowbuf);
        });
}

}  // namespace

size_t mce_smem_bytes(int wpl, int warps_per_block) {
    return (size_t)warps_per_block * (32u * 32u * wpl + 32u * wpl) * sizeof(uint32_t);
}

template <int WPL, bool M>
static void launch_one(const MceArgs &a, dim3 g, dim3 b, size_t sm, cudaStream_t st) {
    if (!M && a.deadline) {  // budgeted runs (never the metrics build)
        cudaFuncSetAttribute(mce_kernel<WPL, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
        mce_kernel<WPL, false, true><<<g, b, sm, st>>>(a);
        return;
    }
    cudaFuncSetAttribute(mce_kernel<WPL, M, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    mce_kernel<WPL, M, false><<<g, b, sm, st>>>(a);
}

template <int WPL, bool M>
static int mce_occ(int warps_per_block) {
    const size_t sm = mce_smem_bytes(WPL, warps_per_block);
    cudaFuncSetAttribute(mce_kernel<WPL, M, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, mce_kernel<WPL, M, false>, 32 * warps_per_block, sm) !=
        cudaSuccess)
        return 0;
    return nb;
}

int mce_blocks_per_sm(int wpl, int warps_per_block, bool metrics) {
    switch (wpl) {
        case 1: return metrics ? mce_occ<1, true>(warps_per_block) : mce_occ<1, false>(warps_per_block);
        case 2: return metrics ? mce_occ<2, true>(warps_per_block) : mce_occ<2, false>(warps_per_block);
        case 4: return metrics ? mce_occ<4, true>(warps_per_block) : mce_occ<4, false>(warps_per_block);
        case 8: return metrics ? mce_occ<8, true>(warps_per_block) : mce_occ<8, false>(warps_per_block);
        default: return 0;
    }
}

__global__ void epoch_bump_kernel(uint32_t *e) {
    uint32_t v = *e + 1u;
    *e = v ? v : 1u;
}

cudaError_t epoch_bump(uint32_t *epoch_dev, cudaStream_t st) {
    epoch_bump_kernel<<<1, 1, 0, st>>>(epoch_dev);
    return cudaGetLastError();
}

__global__ void deadline_set_kernel(unsigned long long *d, unsigned long long budget_ns) {
    unsigned long long now;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    *d = now + budget_ns;
}

cudaError_t deadline_set(unsigned long long *deadline, unsigned long long budget_ns, cudaStream_t st) {
    deadline_set_kernel<<<1, 1, 0, st>>>(deadline, budget_ns);
    return cudaGetLastError();
}

__global__ void flag_left_kernel(const unsigned long long *left, int *status) {
    if (*left) atomicOr(status, kStatusDeferOverflow);
}

cudaError_t flag_left(const unsigned long long *left, int *status, cudaStream_t st) {
    flag_left_kernel<<<1, 1, 0, st>>>(left, status);
    return cudaGetLastError();
}

cudaError_t mce_launch(int wpl, const MceArgs &a, int blocks, int warps_per_block, cudaStream_t st) {
    size_t sm = mce_smem_bytes(wpl, warps_per_block);
    dim3 g(blocks), b(32 * warps_per_block);
    const bool m = a.work != nullptr;
    switch (wpl) {
        case 1: m ? launch_one<1, true>(a, g, b, sm, st) : launch_one<1, false>(a, g, b, sm, st); break;
        case 2: m ? launch_one<2, true>(a, g, b, sm, st) : launch_one<2, false>(a, g, b, sm, st); break;
        case 4: m ? launch_one<4, true>(a, g, b, sm, st) : launch_one<4, false>(a, g, b, sm, st); break;
        case 8: m ? launch_one<8, true>(a, g, b, sm, st) : launch_one<8, false>(a, g, b, sm, st); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace g2
