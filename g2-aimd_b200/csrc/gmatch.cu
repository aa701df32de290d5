// gmatch.cu - plan-driven subgraph enumeration for sm_100a.
//
// Replaces GMatchApp (app_gmatch/gmatch.h:15-736), which materialises every
// partial embedding level by level in BFS buffers, with a persistent kernel:
// each warp pulls a root (the image of matchOrder[0]) from a device atomic
// queue and extends it depth first.  Two paths, chosen per plan:
//
//  * generic (any plan): the candidates of position i are N(M(parent)) with
//    parent = the back neighbour whose image has the least degree (first on
//    ties, app_gmatch/gmatch.h:516-536), filtered by the plan's conditions
//    (<, >, != against earlier positions, :559-588) and by membership in the
//    other back neighbours' lists (:589-601).  The `<` / `>` conditions are
//    also turned into a [lo, hi) window on the sorted neighbour list before the
//    scan, which removes only candidates the filter rejects.  Candidate lists
//    live in the warp's HBM slab and are generated in chunks (the reference's
//    TEMPSIZE chunking, :617-622), so any degree fits.  The last position is
//    counted, never materialised (:602-609); when it has no back neighbour at
//    position k-2 its candidate set is built once per prefix and counted
//    against (the reference's PREFIX strategy, see shared_last_build).  Long walks hand half of their
//    shallowest pending level (window half, candidate batches) or half of a long
//    last-position scan to idle warps through the record queue of
//    g2_handoff.cuh; records resume from a matched prefix.
//  * clique (plans whose every position is adjacent to all earlier ones with
//    images strictly increasing - presets 0, 23-27): every candidate lies in
//    P0 = N(v) ∩ (v, ∞), so the root's P0 adjacency is built once as bitmap
//    rows and the (k-1)-cliques of that local graph are counted with AND +
//    popc.  Roots whose P0 needs more than 32*WPL words, or whose rows do not
//    fit the slab, take the generic path inside the same kernel.
// Both paths count exactly the embeddings the plan admits, so the result equals
// the reference's "Total counts:".
#include <cstdint>

#include "g2_bitrows.cuh"
#include "g2_device.cuh"
#include "g2_handoff.cuh"
#include "g2_kernels.h"

namespace g2 {

namespace {

__device__ __forceinline__ bool cond_ok(uint32_t op, uint32_t w, uint32_t m) {
    return op == G2_COND_LESS_THAN ? w < m : op == G2_COND_LARGER_THAN ? w > m : w != m;
}

// Count returned by a walk that the run's time budget cut short (nothing of it
// is credited).
constexpr unsigned long long kExpired = ~0ull;

// Has the run's time budget (MatchArgs::deadline, %globaltimer ns) run out?
// Warp-uniform; false without a budget.
__device__ __forceinline__ bool match_deadline_passed(const MatchArgs &a) {
    if (!a.deadline) return false;
    unsigned long long now = 0;
    if (lane_id() == 0) asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(now));
    now = __shfl_sync(G2_FULL, now, 0);
    return now > *a.deadline;
}

struct Level {
    uint64_t pos, end;   // scan window in the parent's neighbour list
    uint32_t len, idx;   // materialised chunk
    uint32_t parent;     // position of the parent back neighbour
};

// Set up the scan window of position i given M[0..i-1].  Returns the sum of
// the back neighbours' degrees (one partial embedding's share of the work model).
__device__ uint64_t level_init(const DevPlan &pl, const uint64_t *rp, const uint32_t *ci, const uint32_t *M,
                               uint32_t i, Level &L) {
    uint32_t parent = pl.bn_pos[i][0];
    uint64_t pd = ldg(rp + M[parent] + 1) - ldg(rp + M[parent]);
    uint64_t dsum = pd;
    for (uint32_t j = 1; j < pl.bn_count[i]; j++) {
        uint32_t b = pl.bn_pos[i][j];
        uint64_t d = ldg(rp + M[b] + 1) - ldg(rp + M[b]);
        dsum += d;
        if (d < pd) pd = d, parent = b;
    }
    uint32_t lo = 0, hi = 0xffffffffu;
    bool hi_set = false;
    for (uint32_t c = 0; c < pl.cond_count[i]; c++) {
        uint32_t m = M[pl.cond_pos[i][c]];
        if (pl.cond_op[i][c] == G2_COND_LARGER_THAN) lo = m + 1 > lo ? m + 1 : lo;
        else if (pl.cond_op[i][c] == G2_COND_LESS_THAN) hi = m < hi ? m : hi, hi_set = true;
    }
    uint64_t s = ldg(rp + M[parent]), e = ldg(rp + M[parent] + 1);
    uint64_t ps = s, pe = e;
    if (lane_id() == 0) {
        ps = lo ? lower_bound(ci, s, e, lo) : s;
        pe = hi_set ? lower_bound(ci, ps, e, hi) : e;
    }
    L.pos = __shfl_sync(G2_FULL, ps, 0);
    L.end = __shfl_sync(G2_FULL, pe, 0);
    L.len = 0;
    L.idx = 0;
    L.parent = parent;
    return dsum;
}

// Does w qualify for position i (conditions + other back neighbours)?
__device__ __forceinline__ bool cand_ok(const DevPlan &pl, const uint64_t *rp, const uint32_t *ci, const uint32_t *M,
                                        uint32_t i,
                                        uint32_t parent, uint32_t w) {
    for (uint32_t c = 0; c < pl.cond_count[i]; c++)
        if (!cond_ok(pl.cond_op[i][c], w, M[pl.cond_pos[i][c]])) return false;
    for (uint32_t j = 0; j < pl.bn_count[i]; j++) {
        uint32_t b = pl.bn_pos[i][j];
        if (b == parent) continue;
        if (!contains(ci, ldg(rp + M[b]), ldg(rp + M[b] + 1), w)) return false;
    }
    return true;
}

// First index in [c, stop) of the sorted list ci with ci[index] >= w, found by
// exponential search from c (the previous answer: candidates come in ascending
// order, so a cursor only moves forward).
__device__ __forceinline__ uint64_t gallop(const uint32_t *ci, uint64_t c, uint64_t stop, uint32_t w) {
    if (c >= stop || ldg(ci + c) >= w) return c;
    uint64_t step = 1;
    while (c + step < stop && ldg(ci + c + step) < w) {
        c += step;
        step <<= 1;
    }
    const uint64_t hi = c + step < stop ? c + step : stop;
    return lower_bound(ci, c + 1, hi, w);
}

// Windows of the last position up to this many entries are counted by
// count_last_sliced; longer ones keep the chunked scan, which can hand off.
constexpr uint64_t kSlicedMax = 32ull * 256ull;

// The last position's count over the window [pos, end) of the parent's list:
// every lane takes a contiguous slice of the window and tests its candidates
// against the conditions and the other back neighbours' lists through cursors
// that only move forward (galloping), instead of a full binary search per
// candidate and list.  Per-lane count.
__device__ __noinline__ unsigned long long count_last_sliced(const DevPlan &pl, const uint64_t *rp,
                                                             const uint32_t *ci, const uint32_t *M, uint32_t i,
                                                             uint32_t parent, uint64_t pos, uint64_t end) {
    const uint32_t lane = lane_id();
    const uint64_t per = (end - pos + 31) >> 5;
    const uint64_t lo = pos + (uint64_t)lane * per;
    const uint64_t hi = lo + per < end ? lo + per : end;
    uint64_t cur[G2_MAX_QUERY], stop[G2_MAX_QUERY];
    uint32_t nb = 0;
    for (uint32_t j = 0; j < pl.bn_count[i]; j++) {
        const uint32_t b = pl.bn_pos[i][j];
        if (b == parent) continue;
        cur[nb] = ldg(rp + M[b]);
        stop[nb] = ldg(rp + M[b] + 1);
        nb++;
    }
    unsigned long long c = 0;
    for (uint64_t x = lo; x < hi; x++) {
        const uint32_t w = ldg(ci + x);
        bool ok = true;
        for (uint32_t t = 0; t < pl.cond_count[i] && ok; t++)
            ok = cond_ok(pl.cond_op[i][t], w, M[pl.cond_pos[i][t]]);
        for (uint32_t t = 0; t < nb && ok; t++) {
            cur[t] = gallop(ci, cur[t], stop[t], w);
            ok = cur[t] < stop[t] && ldg(ci + cur[t]) == w;
        }
        c += ok;
    }
    return c;
}

// Shared candidate set of the last position: the reference's PREFIX store
// strategy (system/plan.h:151-172, app_gmatch/gmatch.h:273-509: a position's
// intersection over the back neighbours that precede its previous position is
// computed once and filtered per previous image), applied to the last
// position k-1.  When no back neighbour of k-1 is position k-2, its candidates
// depend on M[0..k-3] alone: the set S is built once per such prefix (the
// least-degree back neighbour's list filtered by the other back neighbours'
// lists and by the conditions against positions before k-2), and each
// candidate c of position k-2 completes |{x in S : x op c}| embeddings for the
// conditions between k-1 and k-2 - one binary search per candidate instead of
// a scan of the last position's window per candidate.
__device__ __forceinline__ bool last_is_shared(const DevPlan &pl) {
    if (pl.k < 3 || pl.bn_count[pl.k - 1] == 0) return false;
    for (uint32_t j = 0; j < pl.bn_count[pl.k - 1]; j++)
        if (pl.bn_pos[pl.k - 1][j] == pl.k - 2) return false;
    return true;
}

constexpr uint32_t kSharedUnbuilt = 0xffffffffu, kSharedTooLarge = 0xfffffffeu;

// Does position k-2 have exactly the last position's candidate set for every
// prefix?  Same back neighbours and the same conditions against every position
// before k-2 (diamonds, presets 9 and 15, stars: the reference's moving_lvl of
// two positions, system/plan.h:340-371).
__device__ __forceinline__ bool last_pair_same_set(const DevPlan &pl) {
    const uint32_t a = pl.k - 2, b = pl.k - 1;
    if (pl.bn_count[a] != pl.bn_count[b]) return false;
    for (uint32_t j = 0; j < pl.bn_count[a]; j++) {
        bool found = false;
        for (uint32_t t = 0; t < pl.bn_count[b]; t++) found |= pl.bn_pos[b][t] == pl.bn_pos[a][j];
        if (!found) return false;
    }
    for (uint32_t p = 0; p < a; p++) {  // conditions against position p: op set of a == op set of b
        uint32_t ma = 0, mb = 0;
        for (uint32_t c = 0; c < pl.cond_count[a]; c++)
            if (pl.cond_pos[a][c] == p) ma |= 1u << pl.cond_op[a][c];
        for (uint32_t c = 0; c < pl.cond_count[b]; c++)
            if (pl.cond_pos[b][c] == p) mb |= 1u << pl.cond_op[b][c];
        if (ma != mb) return false;
    }
    return true;
}

// Build S for M[0..k-3] into out (at most cap entries, ascending); returns its
// length or kSharedTooLarge.  *dsum = sum of the back neighbours' degrees (the
// work model's share of every partial embedding of length k-1).  The window is
// read 32 entries at a time, each tested by binary search in the other back
// neighbours' lists, survivors compacted by a warp scan.
__device__ __noinline__ uint32_t shared_last_build(const DevPlan &pl, const uint64_t *rp, const uint32_t *ci,
                                                   const uint32_t *M, uint32_t *out, uint32_t cap, uint64_t *dsum) {
    const uint32_t i = pl.k - 1, prev = pl.k - 2;
    const uint32_t lane = lane_id();
    uint32_t parent = pl.bn_pos[i][0];
    uint64_t pd = ldg(rp + M[parent] + 1) - ldg(rp + M[parent]);
    uint64_t ds = pd;
    for (uint32_t j = 1; j < pl.bn_count[i]; j++) {
        const uint32_t b = pl.bn_pos[i][j];
        const uint64_t d = ldg(rp + M[b] + 1) - ldg(rp + M[b]);
        ds += d;
        if (d < pd) pd = d, parent = b;
    }
    *dsum = ds;
    uint32_t lo = 0, hi = 0xffffffffu;
    bool hi_set = false;
    for (uint32_t c = 0; c < pl.cond_count[i]; c++) {
        if (pl.cond_pos[i][c] == prev) continue;
        const uint32_t m = M[pl.cond_pos[i][c]];
        if (pl.cond_op[i][c] == G2_COND_LARGER_THAN) lo = m + 1 > lo ? m + 1 : lo;
        else if (pl.cond_op[i][c] == G2_COND_LESS_THAN) hi = m < hi ? m : hi, hi_set = true;
    }
    const uint64_t s = ldg(rp + M[parent]), e = ldg(rp + M[parent] + 1);
    uint64_t ps = s, pe = e;
    if (lane == 0) {
        ps = lo ? lower_bound(ci, s, e, lo) : s;
        pe = hi_set ? lower_bound(ci, ps, e, hi) : e;
    }
    ps = __shfl_sync(G2_FULL, ps, 0);
    pe = __shfl_sync(G2_FULL, pe, 0);
    uint32_t len = 0;
    for (uint64_t x0 = ps; x0 < pe; x0 += 32) {
        const uint64_t x = x0 + lane;
        const uint32_t w = x < pe ? ldg(ci + x) : 0u;
        bool ok = x < pe;
        for (uint32_t c = 0; c < pl.cond_count[i] && ok; c++)
            if (pl.cond_pos[i][c] != prev) ok = cond_ok(pl.cond_op[i][c], w, M[pl.cond_pos[i][c]]);
        for (uint32_t j = 0; j < pl.bn_count[i] && ok; j++) {
            const uint32_t b = pl.bn_pos[i][j];
            if (b != parent) ok = contains(ci, ldg(rp + M[b]), ldg(rp + M[b] + 1), w);
        }
        uint32_t tot;
        const uint32_t pos = warp_scan(ok, tot);
        if (len + tot > cap) return kSharedTooLarge;  // warp-uniform
        if (ok) out[len + pos] = w;
        len += tot;
    }
    __syncwarp();
    return len;
}

// Embeddings completed by the candidates buf[0..n) of position k-2 against
// S[0..ns); with nparts > 1 only candidates of ordinal ord0 + j with
// (ord0 + j) % nparts == part count (a split root's part).  Per-lane count;
// *taken = this lane's candidates of the part.
__device__ __noinline__ unsigned long long shared_last_count(const DevPlan &pl, const uint32_t *Sv, uint32_t ns,
                                                             const uint32_t *buf, uint32_t n, uint32_t ord0,
                                                             uint32_t part, uint32_t nparts, uint32_t *taken) {
    const uint32_t i = pl.k - 1, prev = pl.k - 2;
    bool lt = false, gt = false, ne = false;
    for (uint32_t c = 0; c < pl.cond_count[i]; c++) {
        if (pl.cond_pos[i][c] != prev) continue;
        const uint32_t op = pl.cond_op[i][c];
        lt |= op == G2_COND_LESS_THAN;
        gt |= op == G2_COND_LARGER_THAN;
        ne |= op == G2_COND_NON_EQUAL;
    }
    unsigned long long cnt = 0;
    uint32_t tk = 0;
    for (uint32_t j = lane_id(); j < n; j += 32) {
        if (nparts > 1 && (ord0 + j) % nparts != part) continue;
        tk++;
        const uint32_t w = buf[j];
        uint32_t a = 0, b = ns;  // first index of S with S[a] >= w
        while (a < b) {
            const uint32_t m = (a + b) >> 1;
            if (Sv[m] < w) a = m + 1;
            else b = m;
        }
        const bool in = a < ns && Sv[a] == w;
        const uint32_t lo = gt ? a + (in ? 1u : 0u) : 0u, hi = lt ? a : ns;
        uint32_t c = hi > lo ? hi - lo : 0u;
        if (ne && in && a >= lo && a < hi) c--;
        cnt += c;
    }
    *taken = tk;
    return cnt;
}

// Embeddings completed when position k-2's candidates are S itself (in
// order): candidate j completes |{x in S : x op S[j]}|, an index range; with
// nparts > 1 only ordinals ord0 + j with (ord0 + j) % nparts == part count.
// Per-lane count; *taken = this lane's candidates of the part.
__device__ __noinline__ unsigned long long shared_pair_count(const DevPlan &pl, uint32_t ns, uint32_t ord0,
                                                             uint32_t part, uint32_t nparts, uint32_t *taken) {
    const uint32_t i = pl.k - 1, prev = pl.k - 2;
    bool lt = false, gt = false, ne = false;
    for (uint32_t c = 0; c < pl.cond_count[i]; c++) {
        if (pl.cond_pos[i][c] != prev) continue;
        const uint32_t op = pl.cond_op[i][c];
        lt |= op == G2_COND_LESS_THAN;
        gt |= op == G2_COND_LARGER_THAN;
        ne |= op == G2_COND_NON_EQUAL;
    }
    unsigned long long cnt = 0;
    uint32_t tk = 0;
    for (uint32_t j = lane_id(); j < ns; j += 32) {
        if (nparts > 1 && (ord0 + j) % nparts != part) continue;
        tk++;
        const uint32_t lo = gt ? j + 1 : 0u, hi = lt ? j : ns;
        uint32_t c = hi > lo ? hi - lo : 0u;
        if (ne && j >= lo && j < hi) c--;
        cnt += c;
    }
    *taken = tk;
    return cnt;
}

// Conditions of position i against position p, as a bit set of operators.
__device__ __forceinline__ uint32_t cond_mask(const DevPlan &pl, uint32_t i, uint32_t p) {
    uint32_t m = 0;
    for (uint32_t c = 0; c < pl.cond_count[i]; c++)
        if (pl.cond_pos[i][c] == p) m |= 1u << pl.cond_op[i][c];
    return m;
}

// The 4-cycle plan (preset 1): M1 and M2 neighbours of M0 with M0 < M1 < M2,
// M3 > M0 a neighbour of both (its `!=` conditions are implied by adjacency).
__device__ __forceinline__ bool plan_is_cycle4(const DevPlan &pl) {
    if (pl.k != 4 || pl.bn_count[1] != 1 || pl.bn_count[2] != 1 || pl.bn_count[3] != 2) return false;
    if (pl.bn_pos[1][0] != 0 || pl.bn_pos[2][0] != 0) return false;
    const uint32_t b0 = pl.bn_pos[3][0], b1 = pl.bn_pos[3][1];
    if (!((b0 == 1 && b1 == 2) || (b0 == 2 && b1 == 1))) return false;
    const uint32_t gt = 1u << G2_COND_LARGER_THAN, ne = 1u << G2_COND_NON_EQUAL;
    return cond_mask(pl, 1, 0) == gt && cond_mask(pl, 2, 0) == gt && cond_mask(pl, 2, 1) == gt &&
           cond_mask(pl, 3, 0) == gt && (cond_mask(pl, 3, 1) & ~ne) == 0 && (cond_mask(pl, 3, 2) & ~ne) == 0;
}

// 4-cycles rooted at v for that plan, counted through the opposite vertex:
// every x > v closes C(c_x, 2) of them, c_x = |{y in N(v) : y > v, x in N(y)}|
// (the pair M1 < M2 is any two of those y).  The c_x live in the warp's slab as
// a dense array over id ranges [lo, lo + slab words), filled by atomics from
// the forward neighbours' lists (each list entry visited once) and summed.
// Taken only when that costs less than the walk's per-pair intersections
// (4 x (ids spanned + the forward neighbours' degrees) <= (d - 1) x those
// degrees, d forward neighbours); false leaves the root to the walk.  count = kExpired when the time budget ran out.
__device__ __noinline__ bool cycle4_root(const MatchArgs &a, uint32_t v, uint32_t *S, unsigned long long &count) {
    const uint32_t lane = lane_id();
    const uint64_t *rp = a.rp;
    const uint32_t *ci = a.ci;
    const uint64_t b = ldg(rp + v), e = ldg(rp + v + 1);
    uint64_t fs = b;
    if (lane == 0) fs = lower_bound(ci, b, e, v + 1);
    fs = __shfl_sync(G2_FULL, fs, 0);
    const uint64_t d = e - fs;
    if (d < 2) return false;
    unsigned long long sdeg = 0, xmax = 0;
    for (uint64_t j = fs + lane; j < e; j += 32) {
        const uint32_t y = ldg(ci + j);
        const uint64_t yb = ldg(rp + y), ye = ldg(rp + y + 1);
        sdeg += ye - yb;
        if (ye > yb) {
            const unsigned long long last = ldg(ci + ye - 1);
            xmax = last > xmax ? last : xmax;
        }
    }
    sdeg = warp_sum_u64(sdeg);
    xmax = warp_max_u64(xmax);
    if (xmax <= v) {
        count = 0;
        return true;
    }
    // the walk intersects d (d - 1) / 2 pairs of forward neighbours' lists, about
    // half the mean degree each; this path clears and sums the id span once and
    // adds every list entry once
    const unsigned long long span = xmax - v;
    if (4ull * (span + sdeg) > (d - 1) * sdeg) return false;
    const uint64_t R = a.words_per_warp;
    unsigned long long total = 0;
    for (uint64_t lo = (uint64_t)v + 1; lo <= xmax; lo += R) {
        const uint64_t hi = lo + R <= xmax + 1 ? lo + R : xmax + 1;  // x in [lo, hi)
        const uint32_t len = (uint32_t)(hi - lo);
        for (uint32_t j = lane; j < len; j += 32) S[j] = 0u;
        __syncwarp();
        for (uint64_t t = fs; t < e; t++) {
            if (a.deadline && ((t - fs) & 63u) == 0 && match_deadline_passed(a)) {
                count = kExpired;
                return true;
            }
            const uint32_t y = ldg(ci + t);
            const uint64_t yb = ldg(rp + y), ye = ldg(rp + y + 1);
            uint64_t ws = yb, we = ye;
            if (lane == 0) {
                ws = lower_bound(ci, yb, ye, (uint32_t)lo);
                we = lower_bound(ci, ws, ye, (uint32_t)(hi - 1)) ;
                if (we < ye && ldg(ci + we) == (uint32_t)(hi - 1)) we++;  // entries <= hi - 1
            }
            ws = __shfl_sync(G2_FULL, ws, 0);
            we = __shfl_sync(G2_FULL, we, 0);
            for (uint64_t x = ws + lane; x < we; x += 32) atomicAdd(S + (ldg(ci + x) - (uint32_t)lo), 1u);
        }
        __syncwarp();
        for (uint32_t j = lane; j < len; j += 32) {
            const unsigned long long c = __ldcg(S + j);
            total += c ? c * (c - 1) / 2 : 0ull;
        }
        __syncwarp();  // the sums have read the range before the next one clears it
    }
    count = warp_sum_u64(total);
    return true;
}

// Record layout of a handed-off plan walk (kMatchRecordWords words): the walk
// resumes at position `level` with M[0..level-1]; kind 0 (prefix) initialises
// that level from the plan, kind 1 (window) scans only [pos, end) of its
// parent's list, kind 2 (candidates) takes `ncand` already-filtered candidates.
constexpr uint32_t kRecKind = 2, kRecN = 3, kRecM = 4, kRecPos = 12, kRecEnd = 14, kRecCand = 16;
constexpr uint32_t kRecMaxCand = kMatchRecordWords - kRecCand;
static_assert(kRecMaxCand >= 8, "record layout");
enum : uint32_t { kRecPrefix = 0, kRecWindow = 1, kRecCandidates = 2 };

__device__ __forceinline__ uint64_t ldcg64(const uint32_t *p) {
    return (uint64_t)__ldcg(p) | ((uint64_t)__ldcg(p + 1) << 32);
}

// Write window records for [p0, p1) of position l in `pieces` equal parts.
__device__ __forceinline__ void put_window(uint32_t *rec, uint32_t task, const uint32_t *M, uint32_t l, uint64_t p0,
                                           uint64_t p1) {
    rec[0] = task;
    rec[1] = l;
    rec[kRecKind] = kRecWindow;
    rec[kRecN] = 0;
    for (uint32_t j = 0; j < l; j++) rec[kRecM + j] = M[j];
    rec[kRecPos] = (uint32_t)p0;
    rec[kRecPos + 1] = (uint32_t)(p0 >> 32);
    rec[kRecEnd] = (uint32_t)p1;
    rec[kRecEnd + 1] = (uint32_t)(p1 >> 32);
}

// Hand half of the pending work of the shallowest open level (levels
// base..i) with enough of it to idle warps and keep walking: the upper half of
// its scan window (in up to 4 pieces) and the later half of its materialised
// candidates (kRecMaxCand per record).  Returns false if nothing was handed off;
// *full is set when the record buffer is exhausted.
__device__ __noinline__ bool match_donate(const MatchArgs &a, uint32_t task, const uint32_t *M, Level *Ls,
                                          uint32_t base, uint32_t i, uint32_t *S, uint32_t CH, bool *full) {
    const uint32_t lane = lane_id();
    uint32_t l = base;
    for (; l <= i; l++)
        if (Ls[l].len - Ls[l].idx >= 2 || Ls[l].end > Ls[l].pos + 64) break;
    if (l > i) return false;
    Level &L = Ls[l];
    const uint64_t span = L.end > L.pos + 64 ? L.end - L.pos : 0;
    const uint64_t wcut = L.pos + span / 2;  // the donor keeps [pos, wcut)
    const uint32_t nw = span ? (uint32_t)((span / 2 + 4095u) / 4096u < 4u ? (span / 2 + 4095u) / 4096u : 4u) : 0u;
    const uint32_t rc = L.len - L.idx;
    const uint32_t dc = rc >= 2 ? rc / 2 : 0;  // candidates handed off: the last dc
    const uint32_t nc = (dc + kRecMaxCand - 1) / kRecMaxCand;
    if (nw + nc == 0) return false;
    const unsigned long long k0 = reserve_records(a, nw + nc);
    if (k0 == ~0ull) {
        *full = true;
        return false;
    }
    const uint32_t *buf = S + (uint64_t)(l - 1) * CH;
    const uint32_t c0 = L.len - dc;
    for (uint32_t r = lane; r < nw + nc; r += 32) {
        uint32_t *rec = a.records + (k0 + r) * a.rec_stride;
        if (r < nw) {
            const uint64_t w = L.end - wcut;
            put_window(rec, task, M, l, wcut + w * r / nw, wcut + w * (r + 1) / nw);
        } else {
            const uint32_t q = r - nw, first = c0 + q * kRecMaxCand;
            const uint32_t cnt = dc - q * kRecMaxCand < kRecMaxCand ? dc - q * kRecMaxCand : kRecMaxCand;
            rec[0] = task;
            rec[1] = l;
            rec[kRecKind] = kRecCandidates;
            rec[kRecN] = cnt;
            for (uint32_t j = 0; j < l; j++) rec[kRecM + j] = M[j];
            for (uint32_t j = 0; j < cnt; j++) rec[kRecCand + j] = buf[first + j];
        }
    }
    publish_records(a, k0, k0 + nw + nc);
    if (span) L.end = wcut;
    L.len -= dc;
    return true;
}

// The last position's scan: hand the upper half of [e, end) to idle warps.
__device__ __noinline__ bool match_donate_last(const MatchArgs &a, uint32_t task, const uint32_t *M, uint32_t l,
                                               uint64_t e, Level &L, bool *full) {
    if (L.end <= e + 1024) return false;
    const uint64_t cut = e + (L.end - e) / 2;
    const unsigned long long k0 = reserve_records(a, 1);
    if (k0 == ~0ull) {
        *full = true;
        return false;
    }
    if (lane_id() == 0) put_window(a.records + k0 * a.rec_stride, task, M, l, cut, L.end);
    publish_records(a, k0, k0 + 1);
    L.end = cut;
    return true;
}

// Generic plan-driven walk of a root (rec == nullptr: M[0] = v) or of a handed-off
// record; returns the number of embeddings and adds the work model (4 x
// back-neighbour degrees per partial embedding) to work.
__device__ __noinline__ unsigned long long match_walk(const MatchArgs &a, const DevPlan &pl, uint32_t task, uint32_t v,
                                                     const uint32_t *rec, uint32_t *S, unsigned long long &work,
                                                     uint32_t part, uint32_t nparts, long long c0) {
    const uint32_t k = pl.k;
    const uint32_t lane = lane_id();
    const uint64_t *rp = a.rp;
    const uint32_t *ci = a.ci;
    uint32_t M[G2_MAX_QUERY];
    Level Ls[G2_MAX_QUERY];
    // slab: candidate chunks of positions 1..k-2, then the last position's
    // shared set when the plan has one (and the slab holds 64-entry chunks)
    const bool shared = last_is_shared(pl) && ((a.words_per_warp / (k - 1)) & ~31ull) >= 64;
    const uint32_t nlists = shared ? k - 1 : k > 2 ? k - 2 : 1;
    const uint32_t CH = (uint32_t)((a.words_per_warp / nlists) & ~31ull);
    uint32_t *Sset = S + (uint64_t)(k - 2) * CH;
    uint32_t s_len = kSharedUnbuilt;  // S for the current M[0..k-3]
    uint64_t s_dsum = 0;
    // position k-2's candidates are S itself: counted by index, never scanned,
    // when its level starts with its whole window (k2_full)
    const bool pair = shared && last_pair_same_set(pl);
    bool k2_full = k == 3;
    unsigned long long count = 0;
    if (CH < 64) {  // a chunk must hold at least two warp-widths of candidates
        if (lane == 0) atomicOr(a.status, kStatusStackOverflow);
        return 0;
    }
    uint32_t base = 1;
    if (!rec) {
        M[0] = v;
        const uint64_t w1 = 4ull * level_init(pl, rp, ci, M, 1, Ls[1]);
        if (part == 0) work += w1;
    } else {
        // record words are read past L1 (two records share a cache line)
        base = __ldcg(rec + 1);
        const uint32_t kind = __ldcg(rec + kRecKind);
        k2_full = base == k - 2 && kind == kRecPrefix;
        for (uint32_t j = 0; j < base; j++) M[j] = __ldcg(rec + kRecM + j);
        const uint64_t d = level_init(pl, rp, ci, M, base, Ls[base]);
        if (kind == kRecPrefix) {
            work += 4ull * d;  // this partial embedding's share is counted where it starts
        } else if (kind == kRecWindow) {
            Ls[base].pos = ldcg64(rec + kRecPos);
            Ls[base].end = ldcg64(rec + kRecEnd);
        } else {  // candidates already filtered: they are the level's chunk
            const uint32_t n = __ldcg(rec + kRecN);
            uint32_t *buf = S + (uint64_t)(base - 1) * CH;
            for (uint32_t j = lane; j < n; j += 32) buf[j] = __ldcg(rec + kRecCand + j);
            __syncwarp();
            Ls[base].pos = Ls[base].end = 0;
            Ls[base].len = n;
            Ls[base].idx = 0;
        }
    }
    uint32_t i = base;
    uint32_t ord = 0;  // ordinal of the next position-1 candidate (heavy-root split)
    uint32_t budget_tick = 0;  // time-budget checks every 64 partial embeddings / scan chunks
    bool may_spill = a.spill_cycles != 0 && nparts == 1;
    long long next_check = (long long)a.spill_cycles;
    for (;;) {
        Level &L = Ls[i];
        if (i == k - 1 && L.end - L.pos <= kSlicedMax && !(i == 1 && nparts > 1)) {
            // last position, short window: sliced count with forward-moving cursors
            if (L.pos < L.end) count += warp_sum_u64(count_last_sliced(pl, rp, ci, M, i, L.parent, L.pos, L.end));
            if (i == base) break;
            i--;
            continue;
        }
        if (i == k - 1) {
            // last position: count, never materialise (a long scan hands off its upper half)
            uint32_t iter = 0;
            for (uint64_t e = L.pos; e < L.end; e += 32) {
                if (a.deadline && (++budget_tick & 63u) == 0 && match_deadline_passed(a)) return kExpired;
                if (may_spill && (++iter & 63u) == 0) {
                    long long el = 0;
                    if (lane == 0) el = clock64() - c0;
                    el = __shfl_sync(G2_FULL, el, 0);
                    if (el > next_check) {
                        if (handoff_wanted(a)) {
                            bool full = false;
                            match_donate_last(a, task, M, i, e + 32, L, &full);
                            if (full) may_spill = false;
                        }
                        next_check = el + (long long)a.spill_cycles;
                    }
                }
                uint64_t x = e + lane;
                bool ok = x < L.end && cand_ok(pl, rp, ci, M, i, L.parent, ldg(ci + x));
                uint32_t b = __ballot_sync(G2_FULL, ok);
                if (i == 1 && nparts > 1) {  // k == 2: split the candidates themselves
                    uint32_t keep = 0;
                    for (uint32_t bits = b; bits; bits &= bits - 1)
                        if ((ord++ % nparts) == part) keep |= bits & (~bits + 1u);
                    b = keep;
                }
                count += __popc(b);
            }
            if (i == base) break;
            i--;
            continue;
        }
        if (pair && i == k - 2 && k2_full) {
            k2_full = false;
            if (s_len == kSharedUnbuilt) s_len = shared_last_build(pl, rp, ci, M, Sset, CH, &s_dsum);
            if (s_len != kSharedTooLarge) {
                const bool split = i == 1 && nparts > 1;
                uint32_t tk = 0;
                count += warp_sum_u64(shared_pair_count(pl, s_len, ord, part, split ? nparts : 1u, &tk));
                work += 4ull * s_dsum * warp_sum_u64(tk);
                if (split) ord += s_len;
                L.pos = L.end;  // the level is done
                L.len = L.idx = 0;
                if (a.deadline && match_deadline_passed(a)) return kExpired;
                continue;
            }
        }
        uint32_t *buf = S + (uint64_t)(i - 1) * CH;
        if (L.idx == L.len) {
            if (L.pos >= L.end) {
                if (i == base) break;
                i--;
                continue;
            }
            // next chunk of candidates
            uint32_t len = 0;
            while (L.pos < L.end && len + 32 <= CH) {
                uint64_t x = L.pos + lane;
                uint32_t w = x < L.end ? ldg(ci + x) : 0u;
                bool ok = x < L.end && cand_ok(pl, rp, ci, M, i, L.parent, w);
                uint32_t tot;
                uint32_t pos = warp_scan(ok, tot);
                if (ok) buf[len + pos] = w;
                len += tot;
                L.pos += 32;
            }
            __syncwarp();
            L.len = len;
            L.idx = 0;
            continue;
        }
        auto maybe_donate = [&]() {  // every spill_cycles: hand work to idle warps
            long long el = 0;
            if (lane == 0) el = clock64() - c0;
            el = __shfl_sync(G2_FULL, el, 0);
            if (el > next_check) {
                if (handoff_wanted(a)) {
                    bool full = false;
                    match_donate(a, task, M, Ls, base, i, S, CH, &full);
                    if (full) may_spill = false;
                }
                next_check = el + (long long)a.spill_cycles;
            }
        };
        if (shared && i == k - 2 && s_len != kSharedTooLarge) {
            // the whole chunk against the last position's shared set
            if (s_len == kSharedUnbuilt) s_len = shared_last_build(pl, rp, ci, M, Sset, CH, &s_dsum);
            if (s_len != kSharedTooLarge) {
                const uint32_t n = L.len - L.idx;
                const bool split = i == 1 && nparts > 1;
                uint32_t tk = 0;
                const unsigned long long c =
                    shared_last_count(pl, Sset, s_len, buf + L.idx, n, ord, part, split ? nparts : 1u, &tk);
                count += warp_sum_u64(c);
                work += 4ull * s_dsum * warp_sum_u64(tk);
                if (split) ord += n;
                L.idx = L.len;
                if (a.deadline && match_deadline_passed(a)) return kExpired;
                if (may_spill) maybe_donate();
                continue;
            }
        }
        M[i] = buf[L.idx];
        L.idx++;
        if (a.deadline && (++budget_tick & 63u) == 0 && match_deadline_passed(a)) return kExpired;
        if (i == 1 && nparts > 1 && (ord++ % nparts) != part) continue;  // another part's candidate
        if (may_spill) maybe_donate();
        i++;
        work += 4ull * level_init(pl, rp, ci, M, i, Ls[i]);
        if (i == k - 2) s_len = kSharedUnbuilt, k2_full = true;
    }
    return count;
}

// A root of a non-clique plan (or a clique root whose rows do not fit): the
// 4-cycle count through opposite vertices where that is cheaper, else the walk.
// (Runs with the work model keep the walk: the model counts its steps.)
template <bool METRICS>
__device__ __noinline__ unsigned long long match_root_plan(const MatchArgs &a, const DevPlan &pl, uint32_t task,
                                                           uint32_t v, uint32_t *S, unsigned long long &work,
                                                           uint32_t part, uint32_t nparts, long long c0) {
    unsigned long long c = 0;
    if (!METRICS && nparts == 1 && plan_is_cycle4(pl) && cycle4_root(a, v, S, c)) return c;
    return match_walk(a, pl, task, v, nullptr, S, work, part, nparts, c0);
}

// Bits of word w of the mask {j : j > x}.
__device__ __forceinline__ uint32_t above(uint32_t x, uint32_t w) {
    const uint32_t xw = x >> 5;
    return w > xw ? G2_FULL : w < xw ? 0u : ~((2u << (x & 31u)) - 1u);
}

// Number of (k-1)-cliques of the local graph rows A (p rows x W words) with
// increasing indices, k = 3, 4 or 5, summed over the warp.  Lane l owns the
// first indices x = l, l+32, ... with x % nparts == part.
__device__ unsigned long long clique_count_lanes(const MatchArgs &a, const uint32_t *A, uint32_t p, uint32_t W,
                                                 uint32_t k, uint32_t part, uint32_t nparts) {
    unsigned long long c = 0;
    for (uint32_t x = lane_id(); x - lane_id() < p; x += 32) {  // warp-uniform trip count
        if (a.deadline && match_deadline_passed(a)) return kExpired;
        if (x >= p || (nparts > 1 && x % nparts != part)) continue;
        const uint32_t *ax = A + (uint64_t)x * W;
        if (k == 3) {
            for (uint32_t w = x >> 5; w < W; w++) c += __popc(ax[w] & above(x, w));
            continue;
        }
        for (uint32_t w = x >> 5; w < W; w++) {
            for (uint32_t m = ax[w] & above(x, w); m; m &= m - 1) {
                const uint32_t y = (w << 5) + (uint32_t)(__ffs(m) - 1);
                const uint32_t *ay = A + (uint64_t)y * W;
                if (k == 4) {
                    for (uint32_t w2 = y >> 5; w2 < W; w2++) c += __popc(ax[w2] & ay[w2] & above(y, w2));
                    continue;
                }
                for (uint32_t w2 = y >> 5; w2 < W; w2++) {
                    for (uint32_t m2 = ax[w2] & ay[w2] & above(y, w2); m2; m2 &= m2 - 1) {
                        const uint32_t z = (w2 << 5) + (uint32_t)(__ffs(m2) - 1);
                        const uint32_t *az = A + (uint64_t)z * W;
                        for (uint32_t w3 = z >> 5; w3 < W; w3++) c += __popc(ax[w3] & ay[w3] & az[w3] & above(z, w3));
                    }
                }
            }
        }
    }
    return warp_sum_u64(c);
}

// Clique plans on P0 bitmaps.  Returns false if the root does not fit (caller
// falls back to the generic walk).
template <int WPL, bool METRICS>
__device__ bool match_root_clique(const MatchArgs &a, const DevPlan &pl, uint32_t v, uint32_t *S, uint32_t *p0s,
                                  uint32_t *rowbuf,
                                  unsigned long long &count, unsigned long long &work, uint32_t part,
                                  uint32_t nparts) {
    const uint32_t k = pl.k;
    const uint32_t lane = lane_id();
    const uint64_t *rp = a.rp;
    const uint32_t *ci = a.ci;
    const uint64_t lo = ldg(rp + v), hi = ldg(rp + v + 1);
    count = 0;
    unsigned long long w = (METRICS && part == 0) ? (hi - lo) : 0;  // the root's own partial embedding
    if (lo == hi) {
        work += 4ull * w;
        return true;
    }
    const uint64_t split = lo + ldg(a.fo + v);
    const uint32_t p = (uint32_t)(hi - split);
    if (k == 2 || p == 0 || (!METRICS && p + 1 < k)) {
        // k == 2: every forward neighbour is a match; otherwise no k-clique here
        // (the metrics build still walks short roots to count their partial embeddings)
        if (k == 2) count = nparts > 1 ? (p + nparts - 1 - part) / nparts : p;
        work += 4ull * w;
        return true;
    }
    const uint32_t W = (p + 31u) >> 5;
    if (W > 32u * WPL) return false;
    // slab: [A p*W] [frames (k) * (W + 1)]
    const uint64_t a0 = 0, f0 = (uint64_t)p * W;
    if (f0 + (uint64_t)k * (W + 1) > a.words_per_warp) return false;
    // k <= 5 without metrics: the shared region holds P0's membership filter and
    // hit queue; P0 itself is staged in the region's first half when it fits
    // there (the searches of filter hits then read shared memory), else it stays
    // in its CSR slice in global memory.
    if (!METRICS && k <= 5) {
        const uint32_t half = a.p0_words / 2;
        const bool sh = p <= half;
        if (sh) {
            for (uint32_t i = lane; i < p; i += 32) p0s[i] = ldg(ci + split + i);
            __syncwarp();
        }
        uint32_t *fb = sh ? p0s + half : p0s;
        const uint32_t fw = sh ? a.p0_words - half : a.p0_words;
        if (k == 3) {  // triangles: count forward-neighbourhood edges while scanning
            count = sh ? count_forward_edges_filtered<true>(rp, ci, a.fo, p0s, p, part, nparts, fb, fw)
                       : count_forward_edges_filtered<false>(rp, ci, a.fo, ci + split, p, part, nparts, fb, fw);
            return true;
        }
        // lane-parallel counting: lane takes the depth-1 vertices x = lane, lane+32, ...
        // (in ordinal order, so the split filter is x % nparts) and counts the
        // (k-2)-cliques above x serially; it reads only the upper part of rows.
        if (sh) build_upper_rows_filtered<true>(rp, ci, a.fo, p0s, p, W, S + a0, rowbuf, fb, fw, kLongListMatch);
        else build_upper_rows_filtered<false>(rp, ci, a.fo, ci + split, p, W, S + a0, rowbuf, fb, fw, kLongListMatch);
        __syncwarp();
        count = clique_count_lanes(a, S + a0, p, W, k, part, nparts);
        return true;
    }
    for (uint32_t i = lane; i < p; i += 32) p0s[i] = ldg(ci + split + i);
    __syncwarp();
    build_forward_rows(rp, ci, a.fo, p0s, p, W, S + a0, rowbuf, true, kLongListMatch);
    __syncwarp();
    // C = remaining candidates at the current depth; depth = vertices chosen (v included)
    Row<WPL> C;
#pragma unroll
    for (int s = 0; s < WPL; s++) {
        uint32_t w = lane + 32u * s;
        C.w[s] = w < W ? (w + 1 < W || (p & 31u) == 0 ? G2_FULL : ((1u << (p & 31u)) - 1u)) : 0u;
    }
    uint32_t depth = 1;
    uint32_t ord = 0;  // ordinal of the next depth-1 pick (heavy-root split)
    unsigned long long cnt = 0;
    unsigned long long sdeg[G2_MAX_QUERY];  // degree sum of the chosen vertices per depth (metrics)
    sdeg[1] = hi - lo;
    for (;;) {
        // lowest remaining candidate x
        uint32_t key = 0xffffffffu;
#pragma unroll
        for (int s = WPL - 1; s >= 0; s--)
            if (C.w[s]) key = 32u * (uint32_t)s + lane;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
            uint32_t y = __shfl_xor_sync(G2_FULL, key, o);
            key = y < key ? y : key;
        }
        if (key == 0xffffffffu) {
            if (depth == 1) break;
            depth--;
            row_load(C, S + f0 + (uint64_t)depth * (W + 1), W);
            __syncwarp();
            continue;
        }
        const uint32_t x = key * 32u + (uint32_t)(__ffs(row_word(C, key)) - 1);
#pragma unroll
        for (int s = 0; s < WPL; s++)
            if (lane + 32u * s == key) C.w[s] &= ~(1u << (x & 31u));
        if (depth == 1 && nparts > 1 && (ord++ % nparts) != part) continue;  // another part's branch
        Row<WPL> ax;
        row_load(ax, S + a0 + (uint64_t)x * W, W);
        unsigned long long dx = 0;
        if (METRICS) {
            const uint32_t u = p0s[x];
            dx = ldg(rp + u + 1) - ldg(rp + u);
            w += sdeg[depth] + dx;  // partial embedding of length depth + 1
        }
        if (depth + 2 == k) {
            // children would be the last position: count C ∩ A[x]
            uint32_t c = 0;
#pragma unroll
            for (int s = 0; s < WPL; s++) c += __popc(C.w[s] & ax.w[s]);
            cnt += warp_sum_u64(c);
            continue;
        }
        row_store(C, S + f0 + (uint64_t)depth * (W + 1), W);
        __syncwarp();
#pragma unroll
        for (int s = 0; s < WPL; s++) C.w[s] &= ax.w[s];
        if (METRICS) sdeg[depth + 1] = sdeg[depth] + dx;
        depth++;
    }
    count = cnt;
    work += 4ull * w;
    return true;
}

// MINB: CTAs of 256 threads per SM the register budget is set for (4: 64
// registers; 6: 40 registers and more resident warps, which pays on graphs
// larger than L2 where the rows' loads wait on memory).
template <int WPL, bool METRICS, int MINB>
__global__ void __launch_bounds__(256, MINB) match_kernel(MatchArgs a, int clique_path,
                                                          const __grid_constant__ DevPlan pl) {
    extern __shared__ uint32_t smem[];
    if (a.epoch_dev) a.epoch = *a.epoch_dev;
    const uint32_t wib = threadIdx.x >> 5;
    uint32_t *rowbuf = smem + wib * (32u * WPL + a.p0_words);
    uint32_t *p0s = rowbuf + 32u * WPL;
    const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t *S = a.scratch + gw * a.words_per_warp;
    unsigned long long total = 0, work = 0;
    const bool handoff = a.spill_cycles != 0;
    const unsigned long long ntasks = a.ntasks_dev ? *a.ntasks_dev : a.ntasks;
    auto credit = [&](uint32_t task, unsigned long long c, long long c0) {
        if (c == kExpired) {  // dropped by the time budget: nothing counted, no cost recorded
            if (lane_id() == 0) atomicOr(a.status, kStatusDeadline);
            return;
        }
        total += c;
        if (lane_id() == 0) {
            if (a.root_nodes && c) atomicAdd(reinterpret_cast<unsigned long long *>(a.root_nodes + task), c);
            if (a.root_cost)
                atomicAdd(reinterpret_cast<unsigned long long *>(a.root_cost + task),
                          (unsigned long long)(clock64() - c0));
        }
    };
    for (;;) {
        outstanding_add(a, handoff, 1);
        unsigned long long t0 = grab(a.head, a.chunk);
        if (t0 >= ntasks) {
            outstanding_add(a, handoff, -1);
            break;
        }
        unsigned long long t1 = t0 + a.chunk < ntasks ? t0 + a.chunk : ntasks;
        for (unsigned long long t = t0; t < t1; t++) {
            const uint64_t task = a.task_index ? a.task_index[t] : t;
            const uint32_t v = a.tasks[task];
            const uint32_t tp = a.task_part ? a.task_part[task] : (1u << 16);
            const uint32_t nparts = tp >> 16, part = tp & 0xffffu;
            long long c0 = 0;
            if (lane_id() == 0) c0 = clock64();
            c0 = __shfl_sync(G2_FULL, c0, 0);
            unsigned long long c = 0;
            if (match_deadline_passed(a)) {  // time budget spent: start no new root
                credit((uint32_t)task, kExpired, c0);
                continue;
            }
            if (!clique_path || !match_root_clique<WPL, METRICS>(a, pl, v, S, p0s, rowbuf, c, work, part, nparts))
                c = match_root_plan<METRICS>(a, pl, (uint32_t)task, v, S, work, part, nparts, c0);
            credit((uint32_t)task, c, c0);
        }
        outstanding_add(a, handoff, -1);
    }
    if (handoff)
        run_record_queue(a, [&](unsigned long long h) {
            const uint32_t *rec = a.records + h * a.rec_stride;
            if (__ldcg(rec + 1) == kVoidRecord) return;  // slot of a reservation that did not fit
            long long c0 = 0;
            if (lane_id() == 0) c0 = clock64();
            c0 = __shfl_sync(G2_FULL, c0, 0);
            const uint32_t task = __ldcg(rec);
            const unsigned long long c = match_walk(a, pl, task, 0u, rec, S, work, 0u, 1u, c0);
            credit(task, c, c0);
        });
    if (lane_id() == 0 && total) atomicAdd(a.out, total);
    if (METRICS && lane_id() == 0 && work) atomicAdd(a.work, work);
}

}  // namespace

uint32_t match_p0_words(int wpl, bool clique_path, uint32_t k, bool metrics) {
    if (!clique_path) return 0u;
    return (k <= 5 && !metrics) ? 1024u : 1024u * (uint32_t)wpl;
}

size_t match_smem_bytes(int wpl, int warps_per_block, uint32_t p0_words) {
    return (size_t)warps_per_block * (32u * wpl + p0_words) * sizeof(uint32_t);
}

template <int WPL, bool M, int MINB>
static void launch_match(const DevPlan &pl, const MatchArgs &a, dim3 g, dim3 b, size_t sm, cudaStream_t st,
                         int cp) {
    cudaFuncSetAttribute(match_kernel<WPL, M, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    match_kernel<WPL, M, MINB><<<g, b, sm, st>>>(a, cp, pl);
}

template <int WPL, bool M, int MINB>
static int match_occ(int warps_per_block, uint32_t p0_words) {
    const size_t sm = match_smem_bytes(WPL, warps_per_block, p0_words);
    cudaFuncSetAttribute(match_kernel<WPL, M, MINB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    int nb = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, match_kernel<WPL, M, MINB>, 32 * warps_per_block, sm) !=
        cudaSuccess)
        return 0;
    return nb;
}

// The 40-register build exists for the hot case only: WPL 1, no metrics.
static bool wide_budget(int wpl, bool metrics, int ctas_per_sm) { return ctas_per_sm == 6 && wpl == 1 && !metrics; }

int match_blocks_per_sm(int wpl, int warps_per_block, bool metrics, int ctas_per_sm, uint32_t p0_words) {
    const int w = warps_per_block;
    const uint32_t q = p0_words;
    if (wide_budget(wpl, metrics, ctas_per_sm)) return match_occ<1, false, 6>(w, q);
    switch (wpl) {
        case 1: return metrics ? match_occ<1, true, 4>(w, q) : match_occ<1, false, 4>(w, q);
        case 2: return metrics ? match_occ<2, true, 4>(w, q) : match_occ<2, false, 4>(w, q);
        case 4: return metrics ? match_occ<4, true, 4>(w, q) : match_occ<4, false, 4>(w, q);
        case 8: return metrics ? match_occ<8, true, 4>(w, q) : match_occ<8, false, 4>(w, q);
        default: return 0;
    }
}

cudaError_t match_launch(const DevPlan &plan, const MatchArgs &a, int blocks, int warps_per_block, cudaStream_t st,
                         bool clique_path, int wpl, int ctas_per_sm) {
    size_t sm = match_smem_bytes(wpl, warps_per_block, a.p0_words);
    dim3 g(blocks), b(32 * warps_per_block);
    const int cp = clique_path ? 1 : 0;
    const bool m = a.work != nullptr;
    if (wide_budget(wpl, m, ctas_per_sm)) {
        launch_match<1, false, 6>(plan, a, g, b, sm, st, cp);
        return cudaGetLastError();
    }
    switch (wpl) {
        case 1: m ? launch_match<1, true, 4>(plan, a, g, b, sm, st, cp) : launch_match<1, false, 4>(plan, a, g, b, sm, st, cp); break;
        case 2: m ? launch_match<2, true, 4>(plan, a, g, b, sm, st, cp) : launch_match<2, false, 4>(plan, a, g, b, sm, st, cp); break;
        case 4: m ? launch_match<4, true, 4>(plan, a, g, b, sm, st, cp) : launch_match<4, false, 4>(plan, a, g, b, sm, st, cp); break;
        case 8: m ? launch_match<8, true, 4>(plan, a, g, b, sm, st, cp) : launch_match<8, false, 4>(plan, a, g, b, sm, st, cp); break;
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace g2
