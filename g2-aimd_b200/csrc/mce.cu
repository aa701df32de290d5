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
// A root whose rows or frames do not fit in the warp's slab (or whose p needs
// more than 32*WPL words) is deferred: the host re-runs deferred roots with a
// larger slab per warp (fewer warps) or a wider WPL.  No spin waits exist.
#include <cstdint>

#include "g2_bitrows.cuh"
#include "g2_device.cuh"
#include "g2_kernels.h"

namespace g2 {

namespace {

struct Frame {  // offsets inside the warp slab
    static __device__ __forceinline__ uint32_t size(uint32_t W) { return 3u * W + 2u; }
};

template <int WPL>
__device__ void defer_root(const MceArgs &a, uint64_t t) {
    if (lane_id() == 0) {
        unsigned long long d = atomicAdd(a.ndeferred, 1ull);
        if (d < a.deferred_cap) a.deferred[d] = (uint32_t)t;
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

// Walk one root.  Returns false if the root had to be deferred.  With METRICS
// the work model W (in 4-byte words) of the reference's tree is accumulated:
// per node with P ∪ X non-empty, sum_{u in P∪X} (|P| + deg u) for pivot
// scoring plus sum_{q in P \ N(pivot)} (|P ∪ X| + deg q) for the children.
template <int WPL, bool METRICS>
__device__ bool mce_root(const MceArgs &a, uint64_t t, uint32_t *S, uint32_t *cand, uint32_t *rowbuf) {
    const uint32_t lane = lane_id();
    const uint64_t *rp = a.rp;
    const uint32_t *ci = a.ci;
    const uint32_t v = a.tasks[t];
    const uint64_t lo = ldg(rp + v), hi = ldg(rp + v + 1);
    // heavy-root split: this task owns the root's top-level branches whose ordinal
    // is congruent to part mod nparts (the root record itself belongs to part 0)
    const uint32_t tp = a.task_part ? a.task_part[t] : (1u << 16);
    const uint32_t nparts = tp >> 16, part = tp & 0xffffu;
    if (lo == hi || (part != 0 && ldg(a.fo + v) == hi - lo)) {  // no neighbours (app_BK/BK.h:335-336) or P empty
        if (a.root_nodes && lane == 0) a.root_nodes[t] = 0;
        return true;
    }
    uint32_t branch = 0;  // ordinal of the next top-level branch
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
        if (a.root_nodes && lane == 0) a.root_nodes[t] = 1;
        return true;
    }
    const uint32_t W = (p + 31u) >> 5;
    if (W > 32u * WPL) return false;
    const uint64_t SW = a.words_per_warp;
    const uint32_t FR = Frame::size(W);
    // slab: [hist u64 (p+2)] [A p*W] [xv nx (metrics)] [B nb*W] [lists ...] ... [frames (p+1)*FR]
    const uint64_t h0 = 0, a0 = 2ull * (p + 2), xv0 = a0 + (uint64_t)p * W;
    const uint64_t b0 = xv0 + (METRICS ? nx : 0);  // metrics: X0 vertex of each kept B row
    const uint64_t fr0 = SW >= (uint64_t)(p + 1) * FR ? SW - (uint64_t)(p + 1) * FR : 0;
    if (fr0 < b0 + 64) return false;
    unsigned long long *hist_local = reinterpret_cast<unsigned long long *>(S + h0);
    for (uint32_t s = lane; s < p + 2; s += 32) hist_local[s] = 0ull;
    // ---- stage P0 in shared memory, then the rows
    for (uint32_t i = lane; i < p; i += 32) cand[i] = ldg(ci + split + i);
    __syncwarp();
    build_forward_rows(rp, ci, a.fo, cand, p, W, S + a0, rowbuf);
    uint32_t *Bfull = S + b0;
    // kept B rows plus their root-list entries must stay below the frames
    const uint64_t cap64 = (fr0 - b0 - 64) / (W + 1);
    const uint32_t cap = cap64 > 0xfffffff0ull ? 0xfffffff0u : (uint32_t)cap64;
    const uint32_t nb = build_back_rows(rp, ci, a.fo, v, lo, nx, cand, p, W, Bfull, METRICS ? S + xv0 : nullptr,
                                        cap, rowbuf);
    if (nb == ~0u) return false;
    __syncwarp();
    // ---- root list (identity over the nb kept rows), right after B
    const uint64_t l0 = b0 + (uint64_t)nb * W;
    for (uint32_t i = lane; i < nb; i += 32) S[l0 + i] = i;
    __syncwarp();

    // ---- depth-first walk
    Row<WPL> P, X, Qr;
#pragma unroll
    for (int s = 0; s < WPL; s++) {
        uint32_t w = lane + 32u * s;
        P.w[s] = w < W ? (w + 1 < W || (p & 31u) == 0 ? G2_FULL : ((1u << (p & 31u)) - 1u)) : 0u;
        X.w[s] = 0u;
        Qr.w[s] = 0u;
    }
    uint64_t xoff = l0;
    uint32_t xlen = nb;
    uint32_t d = 0;  // |R| = d + 1
    unsigned long long nodes = 0, cliques = 0, work = 0;
    bool enter = true;
    bool overflow = false;
    for (;;) {
        bool want_pop = false;
        if (enter) {
            enter = false;
            if (d > 0 || part == 0) nodes++;
            uint32_t anyp = 0, anyx = 0;
#pragma unroll
            for (int s = 0; s < WPL; s++) anyp |= P.w[s], anyx |= X.w[s];
            const bool hp = __any_sync(G2_FULL, anyp != 0);
            const bool hx = __any_sync(G2_FULL, anyx != 0) || xlen > 0;
            unsigned long long npx = 0;  // |P| + |X| (metrics)
            if (METRICS && (hp || hx) && (d > 0 || part == 0)) {
                // the reference's root record keeps every X0 vertex, also those
                // with no neighbour in P0 that the B list drops (they fall out of
                // every child), so the root node counts all of X0
                const uint32_t np = row_popc(P);
                npx = np + row_popc(X) + (d == 0 ? nx : xlen);
                unsigned long long sd = row_degree_sum(P, rp, ci, split) + row_degree_sum(X, rp, ci, split);
                unsigned long long sx = 0;
                if (d == 0) {
                    for (uint32_t li = lane; li < nx; li += 32) {
                        const uint32_t u = ldg(ci + lo + li);
                        sx += ldg(rp + u + 1) - ldg(rp + u);
                    }
                } else {
                    for (uint32_t li = lane; li < xlen; li += 32) {
                        const uint32_t u = S[xv0 + S[xoff + li]];
                        sx += ldg(rp + u + 1) - ldg(rp + u);
                    }
                }
                work += npx * np + sd + warp_sum_u64(sx);
            }
            if (!hp) {
                if (!hx) {  // no P and no X: maximal (app_BK/BK.h:78-91)
                    cliques++;
                    if (lane == 0) hist_local[d + 1]++;
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
                    const uint32_t *r = S + a0 + (uint64_t)idx * W;
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
                    rank >= nb ? S + a0 + (uint64_t)(rank - nb) * W : Bfull + (uint64_t)rank * W;
                Row<WPL> pr;
                row_load(pr, prow, W);
#pragma unroll
                for (int s = 0; s < WPL; s++) Qr.w[s] = P.w[s] & ~pr.w[s];
                if (METRICS && (d > 0 || part == 0)) work += npx * row_popc(Qr) + row_degree_sum(Qr, rp, ci, split);
            }
        }
        if (!want_pop) {
            // ---- next branch q of the current node: lowest set bit of Qr
            uint32_t key = 0xffffffffu;
#pragma unroll
            for (int s = WPL - 1; s >= 0; s--)
                if (Qr.w[s]) key = 32u * (uint32_t)s + lane;  // word index lane + 32*s
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) {
                uint32_t y = __shfl_xor_sync(G2_FULL, key, o);
                key = y < key ? y : key;
            }
            if (key == 0xffffffffu) {
                want_pop = true;
            } else {
                const uint32_t qw = key;  // word index
                const uint32_t qword = row_word(Qr, qw);
                const uint32_t q = qw * 32u + (uint32_t)(__ffs(qword) - 1);
                const uint32_t qbit = 1u << (q & 31u);
                // q moves from P to X and is consumed from Q
#pragma unroll
                for (int s = 0; s < WPL; s++)
                    if (lane + 32u * s == qw) {
                        P.w[s] &= ~qbit;
                        X.w[s] |= qbit;
                        Qr.w[s] &= ~qbit;
                    }
                if (d == 0 && nparts > 1 && (branch++ % nparts) != part) continue;  // another part's branch
                const uint64_t coff = xoff + xlen;
                if (coff + xlen > fr0) {  // child list would reach the frames
                    overflow = true;
                    break;
                }
                // save the parent state in frame d
                uint32_t *f = S + fr0 + (uint64_t)d * FR;
                row_store(P, f, W);
                row_store(X, f + W, W);
                row_store(Qr, f + 2 * W, W);
                if (lane == 0) {
                    f[3 * W] = (uint32_t)(xoff - b0);
                    f[3 * W + 1] = xlen;
                }
                // child: P ∩ A[q], X_P0 ∩ A[q], B entries adjacent to q
                Row<WPL> aq;
                row_load(aq, S + a0 + (uint64_t)q * W, W);
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
            xoff = b0 + f[3 * W];
            xlen = f[3 * W + 1];
        }
        __syncwarp();
    }
    if (overflow) return false;
    // ---- commit this root's results
    __syncwarp();
    if (lane == 0) {
        atomicAdd(a.out, cliques);
        if (a.root_nodes) a.root_nodes[t] = nodes;
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
    return true;
}

template <int WPL, bool METRICS>
__global__ void __launch_bounds__(256) mce_kernel(MceArgs a) {
    extern __shared__ uint32_t smem[];
    const uint32_t wib = threadIdx.x >> 5;
    uint32_t *cand = smem + wib * (32u * 32u * WPL + 32u * WPL);
    uint32_t *rowbuf = cand + 32u * 32u * WPL;
    const uint64_t gw = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    uint32_t *S = a.scratch + gw * a.words_per_warp;
    unsigned long long ntasks = a.ntasks;
    if (a.ntasks_dev) {
        ntasks = *a.ntasks_dev;
        if (ntasks > a.deferred_cap) ntasks = a.deferred_cap;
    }
    for (;;) {
        unsigned long long t0 = grab(a.head, a.chunk);
        if (t0 >= ntasks) break;
        unsigned long long t1 = t0 + a.chunk < ntasks ? t0 + a.chunk : ntasks;
        for (unsigned long long t = t0; t < t1; t++) {
            uint64_t task = a.task_index ? a.task_index[t] : t;
            const long long c0 = clock64();
            if (!mce_root<WPL, METRICS>(a, task, S, cand, rowbuf)) defer_root<WPL>(a, task);
            else if (a.root_cost && lane_id() == 0) a.root_cost[task] = (uint64_t)(clock64() - c0);
        }
    }
}

}  // namespace

size_t mce_smem_bytes(int wpl, int warps_per_block) {
    return (size_t)warps_per_block * (32u * 32u * wpl + 32u * wpl) * sizeof(uint32_t);
}

template <int WPL, bool M>
static void launch_one(const MceArgs &a, dim3 g, dim3 b, size_t sm, cudaStream_t st) {
    cudaFuncSetAttribute(mce_kernel<WPL, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    mce_kernel<WPL, M><<<g, b, sm, st>>>(a);
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
