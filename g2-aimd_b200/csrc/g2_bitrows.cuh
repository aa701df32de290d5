// g2_bitrows.cuh - bitmap rows over a root's forward neighbourhood P0.
//
// A row is a W-word bitmap over P0 = N(v) ∩ (v, ∞) (local index = position in
// the sorted CSR slice), distributed across the warp: word w lives in lane
// w % 32, register slot w / 32 (WPL slots, so W <= 32 * WPL).
#pragma once

#include <cstdint>

#include "g2_device.cuh"

namespace g2 {

template <int WPL>
struct Row {
    uint32_t w[WPL];
};

template <int WPL>
__device__ __forceinline__ void row_zero(Row<WPL> &r) {
#pragma unroll
    for (int s = 0; s < WPL; s++) r.w[s] = 0;
}

template <int WPL>
__device__ __forceinline__ bool row_any(const Row<WPL> &r) {
    uint32_t o = 0;
#pragma unroll
    for (int s = 0; s < WPL; s++) o |= r.w[s];
    return __any_sync(G2_FULL, o != 0);
}

template <int WPL>
__device__ __forceinline__ void row_load(Row<WPL> &r, const uint32_t *src, uint32_t W) {
    const uint32_t lane = lane_id();
#pragma unroll
    for (int s = 0; s < WPL; s++) {
        uint32_t w = lane + 32u * s;
        r.w[s] = w < W ? src[w] : 0u;
    }
}

template <int WPL>
__device__ __forceinline__ void row_store(const Row<WPL> &r, uint32_t *dst, uint32_t W) {
    const uint32_t lane = lane_id();
#pragma unroll
    for (int s = 0; s < WPL; s++) {
        uint32_t w = lane + 32u * s;
        if (w < W) dst[w] = r.w[s];
    }
}

// Word `w` of a distributed row, broadcast to all lanes (w uniform).
template <int WPL>
__device__ __forceinline__ uint32_t row_word(const Row<WPL> &r, uint32_t w) {
    uint32_t mine = 0;
#pragma unroll
    for (int s = 0; s < WPL; s++)
        if ((w >> 5) == (uint32_t)s) mine = r.w[s];
    return __shfl_sync(G2_FULL, mine, w & 31u);
}

__device__ __forceinline__ uint32_t ilog2p1(uint64_t x) { return 64u - (uint32_t)__clzll((long long)x); }

// Transpose of a 32x32 bit tile held one word per lane: on return lane L
// holds the word whose bit l is bit L of lane l's input.
__device__ __forceinline__ uint32_t transpose32(uint32_t w) {
    const uint32_t lane = lane_id();
    uint32_t t = 0;
#pragma unroll
    for (int b = 0; b < 32; b++) {
        uint32_t col = __ballot_sync(G2_FULL, (w >> b) & 1u);
        if (lane == (uint32_t)b) t = col;
    }
    return t;
}

// First index in [lo, hi) of the shared-memory array a with a[i] >= key.
__device__ __forceinline__ uint32_t smem_lower_bound(const uint32_t *a, uint32_t lo, uint32_t hi, uint32_t key) {
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// ---------------------------------------------------------------------------
// Membership filter of P0 (clique plans).  About 90 % of the forward-list
// entries a row build scans are not in P0 (on R-MAT s20, 4.2e8 hits in 4.5e9
// scanned entries), so a one-bit-per-hash filter in shared memory rejects most
// of them with one shared load before any search; only filter hits binary-search
// P0, which then stays in global memory (the root's own CSR slice, L1-resident).
// The filter uses 2^fb bits, fb = log2 of about 32 bits per member (at most the
// space given), so its false-positive rate is at most ~3 % for small P0 and
// p / 2^fb for the largest.
struct P0Filter {
    const uint32_t *bits;
    uint32_t shift;  // slot = (y * kFilterMul) >> shift
};
constexpr uint32_t kFilterMul = 0x9E3779B1u;  // Fibonacci hashing

// P0 entry j: from shared memory when P0 is staged there (SH), else from the
// root's CSR slice in global memory.
template <bool SH>
__device__ __forceinline__ uint32_t p0_at(const uint32_t *P0, uint32_t j) {
    if constexpr (SH) return P0[j];
    else return ldg(P0 + j);
}

template <bool SH = false>
__device__ __forceinline__ P0Filter filter_build(uint32_t *bits, uint32_t max_words, const uint32_t *P0, uint32_t p) {
    const uint32_t lane = lane_id();
    uint32_t fb = 10;  // at least 1024 bits
    while (fb < 31 && (1u << fb) < 32u * p && (1u << (fb + 1)) <= 32u * max_words) fb++;
    const uint32_t words = 1u << (fb - 5), shift = 32u - fb;
    for (uint32_t w = lane; w < words; w += 32) bits[w] = 0u;
    __syncwarp();
    for (uint32_t i = lane; i < p; i += 32) {
        const uint32_t h = (p0_at<SH>(P0, i) * kFilterMul) >> shift;
        atomicOr(bits + (h >> 5), 1u << (h & 31u));
    }
    __syncwarp();
    return P0Filter{bits, shift};
}

__device__ __forceinline__ bool filter_maybe(const P0Filter &f, uint32_t y) {
    const uint32_t h = (y * kFilterMul) >> f.shift;
    return (f.bits[h >> 5] >> (h & 31u)) & 1u;
}

// First index in [lo, hi) of P0 with P0[i] >= key (shared or global memory).
template <bool SH>
__device__ __forceinline__ uint32_t p0_lower_bound(const uint32_t *a, uint32_t lo, uint32_t hi, uint32_t key) {
    while (lo < hi) {
        uint32_t mid = (lo + hi) >> 1;
        if (p0_at<SH>(a, mid) < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Forward lists longer than this are scanned by the whole warp (coalesced, one
// row at a time) instead of by their row's lane.  The lane loop runs as long as
// the warp's longest list, so a lower bound balances lanes better; the walks of
// clique plans gain from 32 (R-MAT s20 4-cliques 18.3 -> 17.3 ms), while MCE's
// row builds (more, shorter rows per root) lose below 96.
constexpr uint32_t kLongList = 96;
constexpr uint32_t kLongListMatch = 32;

// Adjacency rows of the root's forward neighbourhood.
//   p0s   : P0 = N(v) ∩ (v, ∞) staged in shared memory (p sorted ids)
//   fo    : fo[u] = offset of the first neighbour of u larger than u
//   A     : p rows of W words (slab), row i = N(P0[i]) ∩ P0
// Upper parts come from forward lists (P0[j] ∈ N+(P0[i]) for j > i), one lane
// per row (the warp together for long lists); the lower parts are the
// transpose, added 32x32 tile by tile.
// With symmetric = false only the upper part of each row (words from i / 32
// on, bits j > i) is built: enough for walks that only look above the row.
__device__ __noinline__ static void build_forward_rows(const uint64_t *rp, const uint32_t *ci, const uint32_t *fo,
                                   const uint32_t *p0s, uint32_t p, uint32_t W, uint32_t *A, uint32_t *rowbuf,
                                   bool symmetric = true, uint32_t long_list = kLongList) {
    const uint32_t lane = lane_id();
    const uint32_t pmax = p0s[p - 1];
    if (symmetric)
        for (uint64_t w = lane; w < (uint64_t)p * W; w += 32) A[w] = 0u;
    else
        for (uint32_t i = lane; i < p; i += 32)
            for (uint32_t w = i >> 5; w < W; w++) A[(uint64_t)i * W + w] = 0u;
    __syncwarp();
    for (uint32_t i0 = 0; i0 < p; i0 += 32) {
        const uint32_t i = i0 + lane;
        bool big = false;
        if (i < p) {
            const uint32_t u = p0s[i];
            uint64_t e = ldg(rp + u) + ldg(fo + u);
            const uint64_t end = ldg(rp + u + 1);
            if (end - e > long_list) big = true;
            else {
                uint32_t *row = A + (uint64_t)i * W;
                uint32_t j = i + 1;
                for (; e < end; e++) {
                    const uint32_t y = ldg(ci + e);
                    if (y > pmax) break;
                    j = smem_lower_bound(p0s, j, p, y);
                    if (j < p && p0s[j] == y) row[j >> 5] |= 1u << (j & 31u);
                }
            }
        }
        uint32_t bigmask = __ballot_sync(G2_FULL, big);
        while (bigmask) {
            const uint32_t l = __ffs(bigmask) - 1;
            bigmask &= bigmask - 1;
            const uint32_t ii = i0 + l;
            const uint32_t u = p0s[ii];
            const uint64_t e0 = ldg(rp + u) + ldg(fo + u), end = ldg(rp + u + 1);
            for (uint32_t w = lane; w < W; w += 32) rowbuf[w] = 0u;
            __syncwarp();
            for (uint64_t e = e0 + lane; e < end; e += 32) {
                const uint32_t y = ldg(ci + e);
                if (y > pmax) break;
                const uint32_t j = smem_lower_bound(p0s, ii + 1, p, y);
                if (j < p && p0s[j] == y) atomicOr(rowbuf + (j >> 5), 1u << (j & 31u));
            }
            __syncwarp();
            for (uint32_t w = lane; w < W; w += 32) A[(uint64_t)ii * W + w] = rowbuf[w];
            __syncwarp();
        }
    }
    __syncwarp();
    if (!symmetric) return;
    // A |= A^T over upper tiles (tr <= tc)
    for (uint32_t tr = 0; tr < W; tr++) {
        for (uint32_t tc = tr; tc < W; tc++) {
            const uint32_t r = 32u * tr + lane;
            const uint32_t w = r < p ? A[(uint64_t)r * W + tc] : 0u;
            const uint32_t t = transpose32(w);
            const uint32_t r2 = 32u * tc + lane;
            if (r2 < p) A[(uint64_t)r2 * W + tr] |= t;
            __syncwarp();
        }
    }
}

// Number of edges of the root's forward neighbourhood (triangles rooted at v)
// with i % nparts == part for the lower end i, counted during the forward-list
// scan without building rows.  Warp total.
__device__ __noinline__ static unsigned long long count_forward_edges(const uint64_t *rp, const uint32_t *ci,
                                                                      const uint32_t *fo, const uint32_t *p0s,
                                                                      uint32_t p, uint32_t part, uint32_t nparts) {
    const uint32_t lane = lane_id();
    const uint32_t pmax = p0s[p - 1];
    unsigned long long c = 0;
    for (uint32_t i0 = 0; i0 < p; i0 += 32) {
        const uint32_t i = i0 + lane;
        bool big = false;
        if (i < p && (nparts <= 1 || i % nparts == part)) {
            const uint32_t u = p0s[i];
            uint64_t e = ldg(rp + u) + ldg(fo + u);
            const uint64_t end = ldg(rp + u + 1);
            if (end - e > kLongListMatch) big = true;
            else {
                uint32_t j = i + 1;
                for (; e < end; e++) {
                    const uint32_t y = ldg(ci + e);
                    if (y > pmax) break;
                    j = smem_lower_bound(p0s, j, p, y);
                    c += j < p && p0s[j] == y;
                }
            }
        }
        uint32_t bigmask = __ballot_sync(G2_FULL, big);
        while (bigmask) {
            const uint32_t l = __ffs(bigmask) - 1;
            bigmask &= bigmask - 1;
            const uint32_t ii = i0 + l;
            const uint32_t u = p0s[ii];
            const uint64_t e0 = ldg(rp + u) + ldg(fo + u), end = ldg(rp + u + 1);
            for (uint64_t e = e0 + lane; e < end; e += 32) {
                const uint32_t y = ldg(ci + e);
                if (y > pmax) break;
                const uint32_t j = smem_lower_bound(p0s, ii + 1, p, y);
                c += j < p && p0s[j] == y;
            }
        }
    }
    return warp_sum_u64(c);
}

// Hits of one long forward list N+(u) = ci[e0, end) in P0[lo, p) (P0 in global
// memory, sorted), found by the whole warp; on_hit(j) runs on some lane for
// every index j with P0[j] in the list.  Two ways, by the cheaper side:
//  * forward: the warp reads the list 32 entries at a time (coalesced), the
//    filter drops most entries, and the survivors are compacted into `queue`
//    (64 words of shared memory) so that every binary search in P0 runs with
//    all 32 lanes busy (without compaction one survivor per 32 entries kept the
//    whole warp searching);
//  * reverse, when |P0[lo, p)| x log |list| is much smaller than the list (a
//    small P0 next to a long list of the dense core): each lane takes P0
//    entries and binary-searches them in the list.
template <bool SH, class F>
__device__ __forceinline__ void warp_list_hits(const uint32_t *ci, uint64_t e0, uint64_t end, const uint32_t *P0,
                                               uint32_t lo, uint32_t p, uint32_t pmax, const P0Filter &f,
                                               uint32_t *queue, F on_hit) {
    const uint32_t lane = lane_id();
    if (lo >= p || e0 >= end) return;
    const uint64_t L = end - e0;  // entries beyond pmax are not scanned, so this bounds the forward cost
    const uint32_t R = p - lo;
    if ((uint64_t)R * (ilog2p1(L) + 1u) * 2u < L) {
        for (uint32_t j = lo + lane; j < p; j += 32) {
            const uint32_t x = p0_at<SH>(P0, j);
            const uint64_t k = lower_bound(ci, e0, end, x);
            if (k < end && ldg(ci + k) == x) on_hit(j);
        }
        return;
    }
    const uint32_t lt = (1u << lane) - 1u;
    uint32_t qn = 0;
    // the next chunk's entry is loaded before this chunk is filtered (its
    // L2 latency overlaps the filter work)
    uint32_t y_next = e0 + lane < end ? ldg(ci + e0 + lane) : 0xffffffffu;
    for (uint64_t base = e0; base < end; base += 32) {
        const uint64_t e = base + lane;
        const uint32_t y = y_next;
        y_next = e + 32 < end ? ldg(ci + e + 32) : 0xffffffffu;
        const bool inr = e < end && y <= pmax;
        if (!__any_sync(G2_FULL, inr)) break;  // sorted: the rest lies beyond P0
        const bool pass = inr && filter_maybe(f, y);
        const uint32_t m = __ballot_sync(G2_FULL, pass);
        if (pass) queue[qn + __popc(m & lt)] = y;
        qn += __popc(m);
        __syncwarp();
        if (qn >= 32) {
            const uint32_t yq = queue[lane];
            const uint32_t jq = p0_lower_bound<SH>(P0, lo, p, yq);
            if (jq < p && p0_at<SH>(P0, jq) == yq) on_hit(jq);
            const uint32_t rest = qn - 32u;
            const uint32_t keep = lane < rest ? queue[32 + lane] : 0u;
            __syncwarp();
            if (lane < rest) queue[lane] = keep;
            qn = rest;
            __syncwarp();
        }
    }
    if (lane < qn) {
        const uint32_t yq = queue[lane];
        const uint32_t jq = p0_lower_bound<SH>(P0, lo, p, yq);
        if (jq < p && p0_at<SH>(P0, jq) == yq) on_hit(jq);
    }
    __syncwarp();
}

// Shared-memory layout of the clique path's per-warp P0 region (fwords words):
// the filter in the first fwords - kQueueWords words, the hit queue after it.
constexpr uint32_t kQueueWords = 64;

// Upper adjacency rows of P0 (row i = bits j > i with P0[j] in N+(P0[i])), as
// build_forward_rows(..., symmetric = false) builds them, with P0 = the root's
// forward slice in global memory and the filter and queue in `fbits` (fwords
// words of shared memory).  One lane per short forward list; lists longer than
// long_list are taken by the whole warp (warp_list_hits) into rowbuf.
template <bool SH>
__device__ __noinline__ static void build_upper_rows_filtered(const uint64_t *rp, const uint32_t *ci,
                                                              const uint32_t *fo, const uint32_t *P0, uint32_t p,
                                                              uint32_t W, uint32_t *A, uint32_t *rowbuf,
                                                              uint32_t *fbits, uint32_t fwords, uint32_t long_list) {
    const uint32_t lane = lane_id();
    const uint32_t pmax = p0_at<SH>(P0, p - 1);
    for (uint32_t i = lane; i < p; i += 32)
        for (uint32_t w = i >> 5; w < W; w++) A[(uint64_t)i * W + w] = 0u;
    uint32_t *queue = fbits + fwords - kQueueWords;
    const P0Filter f = filter_build<SH>(fbits, fwords - kQueueWords, P0, p);
    for (uint32_t i0 = 0; i0 < p; i0 += 32) {
        const uint32_t i = i0 + lane;
        bool big = false;
        if (i < p) {
            const uint32_t u = p0_at<SH>(P0, i);
            uint64_t e = ldg(rp + u) + ldg(fo + u);
            const uint64_t end = ldg(rp + u + 1);
            if (end - e > long_list) big = true;
            else {
                uint32_t *row = A + (uint64_t)i * W;
                uint32_t j = i + 1;
                for (; e < end; e++) {
                    const uint32_t y = ldg(ci + e);
                    if (y > pmax) break;
                    if (!filter_maybe(f, y)) continue;
                    j = p0_lower_bound<SH>(P0, j, p, y);
                    if (j < p && p0_at<SH>(P0, j) == y) row[j >> 5] |= 1u << (j & 31u);
                }
            }
        }
        uint32_t bigmask = __ballot_sync(G2_FULL, big);
        while (bigmask) {
            const uint32_t l = __ffs(bigmask) - 1;
            bigmask &= bigmask - 1;
            const uint32_t ii = i0 + l;
            const uint32_t u = p0_at<SH>(P0, ii);
            const uint64_t e0 = ldg(rp + u) + ldg(fo + u), end = ldg(rp + u + 1);
            for (uint32_t w = lane; w < W; w += 32) rowbuf[w] = 0u;
            __syncwarp();
            warp_list_hits<SH>(ci, e0, end, P0, ii + 1, p, pmax, f, queue,
                           [&](uint32_t j) { atomicOr(rowbuf + (j >> 5), 1u << (j & 31u)); });
            __syncwarp();
            for (uint32_t w = (ii >> 5) + lane; w < W; w += 32) A[(uint64_t)ii * W + w] = rowbuf[w];
            __syncwarp();
        }
    }
    __syncwarp();
}

// count_forward_edges with P0 in global memory and the filter and queue in fbits.
template <bool SH>
__device__ __noinline__ static unsigned long long count_forward_edges_filtered(
    const uint64_t *rp, const uint32_t *ci, const uint32_t *fo, const uint32_t *P0, uint32_t p, uint32_t part,
    uint32_t nparts, uint32_t *fbits, uint32_t fwords) {
    const uint32_t lane = lane_id();
    const uint32_t pmax = p0_at<SH>(P0, p - 1);
    uint32_t *queue = fbits + fwords - kQueueWords;
    const P0Filter f = filter_build<SH>(fbits, fwords - kQueueWords, P0, p);
    unsigned long long c = 0;
    for (uint32_t i0 = 0; i0 < p; i0 += 32) {
        const uint32_t i = i0 + lane;
        bool big = false;
        if (i < p && (nparts <= 1 || i % nparts == part)) {
            const uint32_t u = p0_at<SH>(P0, i);
            uint64_t e = ldg(rp + u) + ldg(fo + u);
            const uint64_t end = ldg(rp + u + 1);
            if (end - e > kLongListMatch) big = true;
            else {
                uint32_t j = i + 1;
                for (; e < end; e++) {
                    const uint32_t y = ldg(ci + e);
                    if (y > pmax) break;
                    if (!filter_maybe(f, y)) continue;
                    j = p0_lower_bound<SH>(P0, j, p, y);
                    c += j < p && p0_at<SH>(P0, j) == y;
                }
            }
        }
        uint32_t bigmask = __ballot_sync(G2_FULL, big);
        while (bigmask) {
            const uint32_t l = __ffs(bigmask) - 1;
            bigmask &= bigmask - 1;
            const uint32_t ii = i0 + l;
            const uint32_t u = p0_at<SH>(P0, ii);
            const uint64_t e0 = ldg(rp + u) + ldg(fo + u), end = ldg(rp + u + 1);
            warp_list_hits<SH>(ci, e0, end, P0, ii + 1, p, pmax, f, queue, [&](uint32_t) { c++; });
        }
    }
    return warp_sum_u64(c);
}

// B rows of the root's backward neighbours X0 = ci[lo, lo+nx) (ids < v):
// row = N+(x) ∩ P0.  Only non-zero rows are kept, compacted in X0 order into
// B (nb rows of W words); xv (optional) receives the vertex of each kept row.
// Returns nb, or ~0u if more than cap rows would be needed.
__device__ __noinline__ static uint32_t build_back_rows(const uint64_t *rp, const uint32_t *ci, const uint32_t *fo, uint32_t v,
                                    uint64_t lo, uint32_t nx, const uint32_t *p0s, uint32_t p, uint32_t W,
                                    uint32_t *B, uint32_t *xv, uint32_t cap, uint32_t *rowbuf) {
    const uint32_t lane = lane_id();
    const uint32_t pmin = p0s[0], pmax = p0s[p - 1];
    uint32_t nb = 0;
    for (uint32_t c = 0; c < nx; c += 32) {
        const uint32_t i = c + lane;
        uint32_t x = 0;
        uint64_t e = 0, end = 0;
        bool hit = false, big = false;
        if (i < nx) {
            x = ldg(ci + lo + i);
            e = ldg(rp + x) + ldg(fo + x);
            end = ldg(rp + x + 1);
            if (end - e > kLongList) big = true;
            else {
                e = lower_bound(ci, e, end, pmin);
                // any element of N+(x) in P0?
                uint32_t j = 0;
                for (uint64_t f = e; f < end; f++) {
                    const uint32_t y = ldg(ci + f);
                    if (y > pmax) break;
                    j = smem_lower_bound(p0s, j, p, y);
                    if (j < p && p0s[j] == y) {
                        hit = true;
                        break;
                    }
                }
            }
        }
        // long lists: decide with the whole warp
        uint32_t bigmask = __ballot_sync(G2_FULL, big);
        uint32_t bighit = 0;
        while (bigmask) {
            const uint32_t l = __ffs(bigmask) - 1;
            bigmask &= bigmask - 1;
            const uint32_t xx = __shfl_sync(G2_FULL, x, l);
            uint64_t b0 = ldg(rp + xx) + ldg(fo + xx), b1 = ldg(rp + xx + 1);
            uint64_t s = 0;
            if (lane == 0) s = lower_bound(ci, b0, b1, pmin);
            s = __shfl_sync(G2_FULL, s, 0);
            bool any = false;
            for (uint64_t base = s; base < b1; base += 32) {  // uniform trip count
                const uint64_t f = base + lane;
                const uint32_t y = f < b1 ? ldg(ci + f) : 0xffffffffu;
                const bool inr = f < b1 && y <= pmax;
                bool found = false;
                if (inr) {
                    const uint32_t j = smem_lower_bound(p0s, 0, p, y);
                    found = j < p && p0s[j] == y;
                }
                if (__any_sync(G2_FULL, found)) {
                    any = true;
                    break;
                }
                if (!__any_sync(G2_FULL, inr)) break;  // sorted: the rest lies beyond P0
            }
            any = __any_sync(G2_FULL, any);
            if (any) bighit |= 1u << l;
        }
        hit = hit || ((bighit >> lane) & 1u);
        uint32_t tot;
        const uint32_t pos = warp_scan(hit, tot);
        if (nb + tot > cap) return ~0u;
        // second pass: write the kept rows at their compacted position
        if (hit && !big) {
            uint32_t *row = B + (uint64_t)(nb + pos) * W;
            for (uint32_t w = 0; w < W; w++) row[w] = 0u;
            uint32_t j = 0;
            for (uint64_t f = e; f < end; f++) {
                const uint32_t y = ldg(ci + f);
                if (y > pmax) break;
                j = smem_lower_bound(p0s, j, p, y);
                if (j < p && p0s[j] == y) row[j >> 5] |= 1u << (j & 31u);
            }
            if (xv) xv[nb + pos] = x;
        }
        uint32_t bm = __ballot_sync(G2_FULL, hit && big);
        while (bm) {
            const uint32_t l = __ffs(bm) - 1;
            bm &= bm - 1;
            const uint32_t xx = __shfl_sync(G2_FULL, x, l);
            const uint32_t dst = nb + __shfl_sync(G2_FULL, pos, l);
            uint64_t b0 = ldg(rp + xx) + ldg(fo + xx), b1 = ldg(rp + xx + 1);
            uint64_t s = 0;
            if (lane == 0) s = lower_bound(ci, b0, b1, pmin);
            s = __shfl_sync(G2_FULL, s, 0);
            for (uint32_t w = lane; w < W; w += 32) rowbuf[w] = 0u;
            __syncwarp();
            for (uint64_t f = s + lane; f < b1; f += 32) {
                const uint32_t y = ldg(ci + f);
                if (y > pmax) break;
                const uint32_t j = smem_lower_bound(p0s, 0, p, y);
                if (j < p && p0s[j] == y) atomicOr(rowbuf + (j >> 5), 1u << (j & 31u));
            }
            __syncwarp();
            for (uint32_t w = lane; w < W; w += 32) B[(uint64_t)dst * W + w] = rowbuf[w];
            if (xv && lane == 0) xv[dst] = xx;
            __syncwarp();
        }
        nb += tot;
        __syncwarp();
    }
    return nb;
}

}  // namespace g2
