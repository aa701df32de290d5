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

constexpr uint32_t kSmallDeg = 128;  // X0 rows built one lane per vertex below this degree

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

// Walk one root.  Returns false if the root had to be deferred.
template <int WPL>
__device__ bool mce_root(const MceArgs &a, uint64_t t, uint32_t *S, uint32_t *cand, uint32_t *rowbuf) {
    const uint32_t lane = lane_id();
    const uint64_t *rp = a.rp;
    const uint32_t *ci = a.ci;
    const uint32_t v = a.tasks[t];
    const uint64_t lo = ldg(rp + v), hi = ldg(rp + v + 1);
    if (lo == hi) {  // no neighbours: skipped, as app_BK/BK.h:335-336
        if (a.root_nodes && lane == 0) a.root_nodes[t] = 0;
        return true;
    }
    uint64_t split = 0;
    if (lane == 0) split = lower_bound(ci, lo, hi, v + 1);
    split = __shfl_sync(G2_FULL, split, 0);
    const uint32_t p = (uint32_t)(hi - split);
    const uint32_t nx = (uint32_t)(split - lo);
    if (p == 0) {  // P empty, X non-empty: one record, not maximal
        if (a.root_nodes && lane == 0) a.root_nodes[t] = 1;
        return true;
    }
    const uint32_t W = (p + 31u) >> 5;
    if (W > 32u * WPL) return false;
    const uint64_t SW = a.words_per_warp;
    const uint32_t FR = Frame::size(W);
    // slab layout: [hist u64 (p+2)] [A p*W] [B nb*W ...] [lists ...] ... [frames (p+1)*FR]
    const uint64_t h0 = 0, a0 = 2ull * (p + 2), b0 = a0 + (uint64_t)p * W;
    const uint64_t fr0 = SW >= (uint64_t)(p + 1) * FR ? SW - (uint64_t)(p + 1) * FR : 0;
    // uncompacted B rows and the root list must fit below the frames
    if (fr0 == 0 || b0 + (uint64_t)nx * W + nx + 64 > fr0) return false;
    unsigned long long *hist_local = reinterpret_cast<unsigned long long *>(S + h0);
    for (uint32_t s = lane; s < p + 2; s += 32) hist_local[s] = 0ull;
    const uint32_t pmax = ldg(ci + hi - 1);

    // ---- A rows
    Row<WPL> row;
    for (uint32_t i = 0; i < p; i++) {
        uint32_t u = ldg(ci + split + i);
        build_row<WPL>(rp, ci, v, split, p, W, pmax, u, row, rowbuf);
        row_store(row, S + a0 + (uint64_t)i * W, W);
    }
    // ---- B rows (uncompacted at b0 + i*W), small-degree X0 vertices one per lane
    uint32_t *Bfull = S + b0;
    for (uint32_t c = 0; c < nx; c += 32) {
        uint32_t i = c + lane;
        bool big = false;
        if (i < nx) {
            uint32_t x = ldg(ci + lo + i);
            uint64_t xlo = ldg(rp + x), xhi = ldg(rp + x + 1);
            uint32_t *r = Bfull + (uint64_t)i * W;
            for (uint32_t w = 0; w < W; w++) r[w] = 0u;
            if (xhi - xlo > kSmallDeg) big = true;
            else {
                uint64_t e = lower_bound(ci, xlo, xhi, v + 1);
                for (; e < xhi; e++) {
                    uint32_t y = ldg(ci + e);
                    if (y > pmax) break;
                    uint64_t j = lower_bound(ci, split, split + p, y);
                    if (j < split + p && ldg(ci + j) == y) {
                        uint32_t jj = (uint32_t)(j - split);
                        r[jj >> 5] |= 1u << (jj & 31u);
                    }
                }
            }
        }
        uint32_t bigmask = __ballot_sync(G2_FULL, big);
        __syncwarp();
        while (bigmask) {
            uint32_t l = __ffs(bigmask) - 1;
            bigmask &= bigmask - 1;
            uint32_t ii = c + l;
            uint32_t x = ldg(ci + lo + ii);
            build_row<WPL>(rp, ci, v, split, p, W, pmax, x, row, rowbuf);
            row_store(row, Bfull + (uint64_t)ii * W, W);
        }
        __syncwarp();
    }
    // compact non-zero B rows in place (destination index <= source index)
    uint32_t nb = 0;
    for (uint32_t i = 0; i < nx; i++) {
        row_load(row, Bfull + (uint64_t)i * W, W);
        if (row_any(row)) {
            if (nb != i) {
                __syncwarp();
                row_store(row, Bfull + (uint64_t)nb * W, W);
            }
            nb++;
        }
        __syncwarp();
    }
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
    unsigned long long nodes = 0, cliques = 0;
    bool enter = true;
    bool overflow = false;
    for (;;) {
        bool want_pop = false;
        if (enter) {
            enter = false;
            nodes++;
            uint32_t anyp = 0, anyx = 0;
#pragma unroll
            for (int s = 0; s < WPL; s++) anyp |= P.w[s], anyx |= X.w[s];
            const bool hp = __any_sync(G2_FULL, anyp != 0);
            const bool hx = __any_sync(G2_FULL, anyx != 0) || xlen > 0;
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
    }
    for (uint32_t s = lane; s < p + 2; s += 32) {
        unsigned long long h = hist_local[s];
        if (h) {
            if (s < a.hist_len) atomicAdd(a.out + 1 + s, h);
            else atomicOr(a.status, kStatusHistOverflow);
        }
    }
    __syncwarp();
    return true;
}

template <int WPL>
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
            if (!mce_root<WPL>(a, task, S, cand, rowbuf)) defer_root<WPL>(a, task);
        }
    }
}

}  // namespace

size_t mce_smem_bytes(int wpl, int warps_per_block) {
    return (size_t)warps_per_block * (32u * 32u * wpl + 32u * wpl) * sizeof(uint32_t);
}

cudaError_t mce_launch(int wpl, const MceArgs &a, int blocks, int warps_per_block, cudaStream_t st) {
    size_t sm = mce_smem_bytes(wpl, warps_per_block);
    dim3 g(blocks), b(32 * warps_per_block);
    switch (wpl) {
        case 1:
            cudaFuncSetAttribute(mce_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            mce_kernel<1><<<g, b, sm, st>>>(a);
            break;
        case 2:
            cudaFuncSetAttribute(mce_kernel<2>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            mce_kernel<2><<<g, b, sm, st>>>(a);
            break;
        case 4:
            cudaFuncSetAttribute(mce_kernel<4>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            mce_kernel<4><<<g, b, sm, st>>>(a);
            break;
        case 8:
            cudaFuncSetAttribute(mce_kernel<8>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
            mce_kernel<8><<<g, b, sm, st>>>(a);
            break;
        default:
            return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

}  // namespace g2
