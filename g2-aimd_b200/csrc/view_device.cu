// view_device.cu - views of a host CSR built by the GPU (G2_VIEW_DEVICE).
//
// The out-of-core pipeline of view_run.cu builds each bin's view on host
// threads (csrc/host/view_host.cpp) and uploads it; for radius-1 views (MCE,
// triangles, k-cliques) the host build is the bound of a call (R-MAT s20 K4:
// 190 ms of building for 18 ms of enumeration).  Here the GPU builds the same
// view directly into its device slot, reading the host CSR through mapped
// (zero-copy) pinned memory:
//   1. sources: degree >= min_deg (order kept), marked in an n-bit bitmap;
//   2. ball: each kept source's row (above the source for upper views) marks
//      its entries in the bitmap;
//   3. local ids: ascending global order = rank in the bitmap (per-word
//      population prefix); the ball list is the bitmap's set bits in order;
//   4. rows: every ball vertex's row restricted to the ball (forward views:
//      entries above the vertex; otherwise from the ball's smallest vertex on),
//      copied once from host memory into a device staging area, then counted
//      (degree, entries <= the vertex) and written as local ids (warp ballots
//      keep the order), row pointers by a scan;
//   5. sources as local ids.
// The result is byte for byte the host builder's (same Layout, same rp, fo, ci,
// src) for shapes with radius 1 and row radius 1 without ego rows.
#include <cub/cub.cuh>

#include <algorithm>
#include <cstdint>
#include <cstring>

#include "host/view_host.h"
#include "runtime_internal.h"
#include "view_device.h"

using namespace g2rt;

namespace {

constexpr uint64_t kLongRow = 256;  // rows longer than this find their start by binary search
constexpr uint64_t kStageMax = 1ull << 29;  // row entries staged in device memory per view (2 GiB)

__device__ __forceinline__ uint32_t lane_of() { return threadIdx.x & 31u; }

// First index in [lo, hi) of the sorted host row with ci[i] >= key.
__device__ __forceinline__ uint64_t row_lower_bound(const uint32_t *ci, uint64_t lo, uint64_t hi, uint32_t key) {
    while (lo < hi) {
        const uint64_t mid = lo + ((hi - lo) >> 1);
        if (ci[mid] < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

// Where row x's scan starts: the first entry >= from (warp-uniform).  Short rows
// start at their beginning (their entries below `from` are skipped while
// streaming); long rows search for it (lane 0) to save the host-memory reads.
__device__ __forceinline__ uint64_t row_start(const uint64_t *rp, const uint32_t *ci, uint32_t x, uint32_t from,
                                              uint64_t *end) {
    const uint64_t b = rp[x], e = rp[x + 1];
    *end = e;
    if (from == 0 || e - b <= kLongRow) return b;
    uint64_t s = 0;
    if (lane_of() == 0) s = row_lower_bound(ci, b, e, from);
    return __shfl_sync(0xffffffffu, s, 0);
}

__device__ __forceinline__ bool bit_of(const uint32_t *bits, uint32_t x) { return (bits[x >> 5] >> (x & 31u)) & 1u; }

// Row of ball vertex i (global id g): from the device staging copy when there is
// one (srp indexed by i, the row already cut at its start), else from the host CSR.
__device__ __forceinline__ const uint32_t *ball_row(const uint64_t *rp, const uint32_t *ci, const uint64_t *srp,
                                                    const uint32_t *sci, uint64_t i, uint32_t g, uint32_t from,
                                                    uint64_t *b, uint64_t *end) {
    if (srp) {
        *b = srp[i];
        *end = srp[i + 1];
        return sci;
    }
    *b = row_start(rp, ci, g, from, end);
    return ci;
}

// A warp per ball vertex: where its row's scan starts in the host CSR, and its length.
__global__ void row_span_kernel(const uint64_t *rp, const uint32_t *ci, const uint32_t *ball, uint64_t nv,
                                bool forward, uint64_t *start, unsigned long long *len) {
    const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t lo = nv ? ball[0] : 0u;
    for (uint64_t i = w0; i < nv; i += nw) {
        const uint32_t g = ball[i];
        uint64_t end;
        const uint64_t b = row_start(rp, ci, g, forward ? g + 1 : lo, &end);
        if (lane_of() == 0) {
            start[i] = b;
            len[i] = end - b;
        }
    }
}

// A warp per ball vertex: its row from the host CSR into the device staging copy
// (the one pass over host memory).
__global__ void row_stage_kernel(const uint32_t *ci, const uint64_t *start, const uint64_t *soff, uint64_t nv,
                                 uint32_t *sci) {
    const uint32_t lane = lane_of();
    const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = w0; i < nv; i += nw) {
        const uint64_t b = start[i], o = soff[i], l = soff[i + 1] - o;
        for (uint64_t k = lane; k < l; k += 32) sci[o + k] = ci[b + k];
    }
}

// Rank of a set bit x in the bitmap: its local id.
__device__ __forceinline__ uint32_t rank_of(const uint32_t *bits, const uint32_t *pre, uint32_t x) {
    return pre[x >> 5] + __popc(bits[x >> 5] & ((1u << (x & 31u)) - 1u));
}

__global__ void keep_sources_kernel(const uint64_t *rp, const uint32_t *roots, uint64_t nroots, uint32_t min_deg,
                                    uint32_t *keep, uint32_t *bits) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nroots; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = roots[i];
        const bool k = rp[s + 1] - rp[s] >= min_deg;
        keep[i] = k;
        if (k) atomicOr(bits + (s >> 5), 1u << (s & 31u));
    }
}

__global__ void compact_sources_kernel(const uint32_t *roots, const uint32_t *keep, const uint32_t *pos,
                                       uint64_t nroots, uint32_t *kept) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < nroots; i += (uint64_t)gridDim.x * blockDim.x)
        if (keep[i]) kept[pos[i]] = roots[i];
}

// A warp per kept source: its row's entries (above the source for upper views)
// join the ball.
__global__ void walk_kernel(const uint64_t *rp, const uint32_t *ci, const uint32_t *kept, uint64_t nkept, bool upper,
                            uint32_t *bits) {
    const uint32_t lane = lane_of();
    const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t k = w0; k < nkept; k += nw) {
        const uint32_t s = kept[k];
        uint64_t end;
        const uint64_t b = row_start(rp, ci, s, upper ? s + 1 : 0u, &end);
        for (uint64_t e = b + lane; e < end; e += 32) {
            const uint32_t u = ci[e];
            if (upper && u <= s) continue;
            atomicOr(bits + (u >> 5), 1u << (u & 31u));
        }
    }
}

__global__ void word_pop_kernel(const uint32_t *bits, uint64_t words, uint32_t *cnt) {
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += (uint64_t)gridDim.x * blockDim.x)
        cnt[w] = __popc(bits[w]);
}

__global__ void ball_list_kernel(const uint32_t *bits, const uint32_t *pre, uint64_t words, uint32_t *ball) {
    for (uint64_t w = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; w < words; w += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t x = bits[w], i = pre[w];
        while (x) {
            ball[i++] = (uint32_t)(w * 32u) + (uint32_t)(__ffs(x) - 1);
            x &= x - 1;
        }
    }
}

// A warp per ball vertex: degree inside the ball and entries <= the vertex.
__global__ void row_count_kernel(const uint64_t *rp, const uint32_t *ci, const uint64_t *srp, const uint32_t *sci,
                                 const uint32_t *ball, uint64_t nv, const uint32_t *bits, bool forward,
                                 unsigned long long *deg, uint32_t *fo, unsigned int *max_fwd) {
    const uint32_t lane = lane_of();
    const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t lo = nv ? ball[0] : 0u;
    for (uint64_t i = w0; i < nv; i += nw) {
        const uint32_t g = ball[i];
        const uint32_t from = forward ? g + 1 : lo;
        uint64_t b, end;
        const uint32_t *row = ball_row(rp, ci, srp, sci, i, g, from, &b, &end);
        uint32_t d = 0, back = 0;
        for (uint64_t e = b + lane; e < end; e += 32) {
            const uint32_t u = row[e];
            if (u < from || !bit_of(bits, u)) continue;
            d++;
            back += u <= g;
        }
        for (int o = 16; o > 0; o >>= 1) {
            d += __shfl_xor_sync(0xffffffffu, d, o);
            back += __shfl_xor_sync(0xffffffffu, back, o);
        }
        if (lane == 0) {
            deg[i] = d;
            fo[i] = back;
            atomicMax(max_fwd, d - back);
        }
    }
}

// A warp per ball vertex: its kept entries as local ids, in order.
__global__ void row_write_kernel(const uint64_t *rp, const uint32_t *ci, const uint64_t *srp, const uint32_t *sci,
                                 const uint32_t *ball, uint64_t nv, const uint32_t *bits, const uint32_t *pre,
                                 bool forward, const uint64_t *vrp, uint32_t *vci) {
    const uint32_t lane = lane_of();
    const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const uint32_t lo = nv ? ball[0] : 0u;
    for (uint64_t i = w0; i < nv; i += nw) {
        uint64_t o = vrp[i];
        if (vrp[i + 1] == o) continue;
        const uint32_t g = ball[i];
        const uint32_t from = forward ? g + 1 : lo;
        uint64_t b, end;
        const uint32_t *row = ball_row(rp, ci, srp, sci, i, g, from, &b, &end);
        for (uint64_t base = b; base < end; base += 32) {
            const uint64_t e = base + lane;
            const uint32_t u = e < end ? row[e] : 0u;
            const bool keep = e < end && u >= from && bit_of(bits, u);
            const uint32_t m = __ballot_sync(0xffffffffu, keep);
            if (keep) vci[o + __popc(m & ((1u << lane) - 1u))] = rank_of(bits, pre, u);
            o += __popc(m);
        }
    }
}

__global__ void src_local_kernel(const uint32_t *kept, uint64_t nkept, const uint32_t *bits, const uint32_t *pre,
                                 uint32_t *src) {
    for (uint64_t k = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; k < nkept; k += (uint64_t)gridDim.x * blockDim.x)
        src[k] = rank_of(bits, pre, kept[k]);
}

// Exclusive scan of n 32-bit counts (CUB; int item count), scratch grown as needed.
template <class T, class U>
cudaError_t scan(const T *in, U *out, uint64_t n, void **tmp, size_t *cap, cudaStream_t st) {
    size_t need = 0;
    cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, need, in, out, (int)n, st);
    if (e != cudaSuccess) return e;
    if (need > *cap) {
        cudaFree(*tmp);
        *tmp = nullptr;
        *cap = 0;
        if ((e = cudaMalloc(tmp, need)) != cudaSuccess) return e;
        *cap = need;
    }
    return cub::DeviceScan::ExclusiveSum(*tmp, need, in, out, (int)n, st);
}

}  // namespace

namespace g2rt {

int DeviceViewBuilder::init(g2_ctx *c, const uint64_t *host_rp, const uint32_t *host_ci, uint64_t nv_graph,
                            const g2view::Shape &shape) {
    ctx = c;
    n = nv_graph;
    sh = shape;
    const uint64_t m = host_rp[n];
    // The host CSR seen from the device: pinned and mapped memory (cudaHostAlloc,
    // a pinning allocator) is used in place; other memory is registered for the
    // call, the arrays' exact byte ranges (one range spanning both if they
    // share a page), else copied once into mapped pinned staging buffers.  Exact
    // ranges matter: the driver counts a registered range as pinned memory, so
    // a range rounded out to whole pages would take in the neighbouring heap
    // blocks, and a pageable copy to or from a block that starts inside the
    // range and ends past it is refused (cudaErrorInvalidValue).
    auto mapped = [](const void *p) -> const void * {
        cudaPointerAttributes at{};
        if (cudaPointerGetAttributes(&at, p) == cudaSuccess && at.type == cudaMemoryTypeHost && at.devicePointer)
            return at.devicePointer;
        cudaGetLastError();
        return nullptr;
    };
    const void *drp = mapped(host_rp), *dci = m ? mapped(host_ci) : host_ci;
    if (!drp || !dci) {
        const uint64_t pg = 4096;
        auto page = [&](uintptr_t a) { return a & ~(uintptr_t)(pg - 1); };
        const uintptr_t a0 = (uintptr_t)host_rp, a1 = a0 + 8 * (n + 1);
        const uintptr_t b0 = m ? (uintptr_t)host_ci : a0, b1 = m ? b0 + 4 * m : a1;
        bool ok = true;
        if (page(b0) <= page(a1 - 1) && page(a0) <= page(b1 - 1)) {  // a page in common: one range
            const uintptr_t u0 = std::min(a0, b0), u1 = std::max(a1, b1);
            ok = cudaHostRegister((void *)u0, u1 - u0, cudaHostRegisterMapped) == cudaSuccess;
            if (ok) reg[nreg++] = (void *)u0;
        } else {
            ok = cudaHostRegister((void *)a0, a1 - a0, cudaHostRegisterMapped) == cudaSuccess;
            if (ok) reg[nreg++] = (void *)a0;
            if (ok && m) {
                ok = cudaHostRegister((void *)b0, b1 - b0, cudaHostRegisterMapped) == cudaSuccess;
                if (ok) reg[nreg++] = (void *)b0;
            }
        }
        void *d = nullptr;
        if (ok) ok = cudaHostGetDevicePointer(&d, const_cast<uint64_t *>(host_rp), 0) == cudaSuccess;
        if (ok) drp = d;
        if (ok && m) {
            ok = cudaHostGetDevicePointer(&d, const_cast<uint32_t *>(host_ci), 0) == cudaSuccess;
            if (ok) dci = d;
        }
        if (!ok) {  // staging copies
            cudaGetLastError();
            for (int k = 0; k < nreg; k++) cudaHostUnregister(reg[k]);
            nreg = 0;
            G2_TRY(cudaHostAlloc(&stage_rp, 8 * (n + 1), cudaHostAllocMapped));
            memcpy(stage_rp, host_rp, 8 * (n + 1));
            G2_TRY(cudaHostGetDevicePointer(&d, stage_rp, 0));
            drp = d;
            if (m) {
                G2_TRY(cudaHostAlloc(&stage_ci, 4 * m, cudaHostAllocMapped));
                memcpy(stage_ci, host_ci, 4 * m);
                G2_TRY(cudaHostGetDevicePointer(&d, stage_ci, 0));
                dci = d;
            }
        }
    }
    hrp = static_cast<const uint64_t *>(drp);
    hci = static_cast<const uint32_t *>(dci);
    words = (n + 31) / 32;
    if (n_cap < std::max<uint64_t>(n, 1) || !bits) {
        for (void *p : {(void *)bits, (void *)wcnt, (void *)wpre, (void *)ball}) cudaFree(p);
        bits = wcnt = wpre = ball = nullptr;
        n_cap = 0;
        const uint64_t w = (std::max<uint64_t>(n, 1) + 31) / 32;
        G2_TRY(cudaMalloc(&bits, 4 * (w + 1)));
        G2_TRY(cudaMalloc(&wcnt, 4 * (w + 1)));
        G2_TRY(cudaMalloc(&wpre, 4 * (w + 1)));
        G2_TRY(cudaMalloc(&ball, 4 * std::max<uint64_t>(n, 1)));
        n_cap = std::max<uint64_t>(n, 1);
    }
    if (!scalars) G2_TRY(cudaMalloc(&scalars, 64));
    return G2_OK;
}

int DeviceViewBuilder::grow_roots(uint64_t need) {
    if (need <= roots_cap) return G2_OK;
    cudaFree(d_roots);
    cudaFree(keep);
    cudaFree(pos);
    cudaFree(kept);
    d_roots = keep = pos = kept = nullptr;
    roots_cap = 0;
    G2_TRY(cudaMalloc(&d_roots, 4 * (need + 1)));
    G2_TRY(cudaMalloc(&keep, 4 * (need + 1)));
    G2_TRY(cudaMalloc(&pos, 4 * (need + 1)));
    G2_TRY(cudaMalloc(&kept, 4 * (need + 1)));
    roots_cap = need;
    return G2_OK;
}

int DeviceViewBuilder::grow_rows(uint64_t need) {
    if (need <= rows_cap) return G2_OK;
    cudaFree(deg);
    cudaFree(fo);
    cudaFree(vrp);
    cudaFree(sstart);
    cudaFree(soff);
    deg = nullptr;
    fo = nullptr;
    vrp = sstart = soff = nullptr;
    rows_cap = 0;
    G2_TRY(cudaMalloc(&deg, 8 * (need + 1)));
    G2_TRY(cudaMalloc(&fo, 4 * (need + 1)));
    G2_TRY(cudaMalloc(&vrp, 8 * (need + 1)));
    G2_TRY(cudaMalloc(&sstart, 8 * (need + 1)));
    G2_TRY(cudaMalloc(&soff, 8 * (need + 1)));
    rows_cap = need;
    return G2_OK;
}

int DeviceViewBuilder::build(const uint32_t *roots, uint64_t nroots, void **buf, uint64_t *cap, cudaStream_t st,
                             g2view::Sizes *out) {
    const int G = ctx->sm_count * 8;
    int rc = grow_roots(std::max<uint64_t>(nroots, 1));
    if (rc) return rc;
    G2_TRY(cudaMemsetAsync(bits, 0, 4 * (words + 1), st));
    G2_TRY(cudaMemsetAsync(scalars, 0, 64, st));
    G2_TRY(cudaMemcpyAsync(d_roots, roots, 4 * nroots, cudaMemcpyHostToDevice, st));
    // 1. sources
    keep_sources_kernel<<<G, 256, 0, st>>>(hrp, d_roots, nroots, sh.min_deg, keep, bits);
    if (nroots) G2_TRY(scan(keep, pos, nroots, &cub_tmp, &cub_cap, st));
    compact_sources_kernel<<<G, 256, 0, st>>>(d_roots, keep, pos, nroots, kept);
    uint32_t nk = 0;
    if (nroots) {
        uint32_t lastk = 0, lastp = 0;
        G2_TRY(cudaMemcpyAsync(&lastk, keep + nroots - 1, 4, cudaMemcpyDeviceToHost, st));
        G2_TRY(cudaMemcpyAsync(&lastp, pos + nroots - 1, 4, cudaMemcpyDeviceToHost, st));
        G2_TRY(cudaStreamSynchronize(st));
        nk = lastp + lastk;
    }
    // 2. ball
    if (nk) walk_kernel<<<G, 256, 0, st>>>(hrp, hci, kept, nk, sh.upper, bits);
    // 3. local ids
    word_pop_kernel<<<G, 256, 0, st>>>(bits, words, wcnt);
    G2_TRY(cudaMemsetAsync(wcnt + words, 0, 4, st));
    G2_TRY(scan(wcnt, wpre, words + 1, &cub_tmp, &cub_cap, st));
    uint32_t nv = 0;
    G2_TRY(cudaMemcpyAsync(&nv, wpre + words, 4, cudaMemcpyDeviceToHost, st));
    G2_TRY(cudaStreamSynchronize(st));
    rc = grow_rows(std::max<uint64_t>(nv, 1));
    if (rc) return rc;
    ball_list_kernel<<<G, 256, 0, st>>>(bits, wpre, words, ball);
    // 4. rows: staged once into device memory (up to kStageMax entries; the
    //    row count and row write then read them there), counts, row pointers,
    //    then columns
    const uint64_t *srp = nullptr;
    const uint32_t *sci = nullptr;
    if (nv) {
        row_span_kernel<<<G, 256, 0, st>>>(hrp, hci, ball, nv, sh.forward, sstart, deg);
        G2_TRY(cudaMemsetAsync(deg + nv, 0, 8, st));
        G2_TRY(scan(deg, soff, (uint64_t)nv + 1, &cub_tmp, &cub_cap, st));
        uint64_t T = 0;
        G2_TRY(cudaMemcpyAsync(&T, soff + nv, 8, cudaMemcpyDeviceToHost, st));
        G2_TRY(cudaStreamSynchronize(st));
        if (T <= kStageMax) {
            if (T > stage_cap) {
                cudaFree(stage);
                stage = nullptr;
                stage_cap = 0;
                G2_TRY(cudaMalloc(&stage, 4 * std::max<uint64_t>(T, 1)));
                stage_cap = T;
            }
            row_stage_kernel<<<G, 256, 0, st>>>(hci, sstart, soff, nv, stage);
            srp = soff;
            sci = stage;
        }
    }
    auto *mx = reinterpret_cast<unsigned int *>(scalars);
    if (nv) row_count_kernel<<<G, 256, 0, st>>>(hrp, hci, srp, sci, ball, nv, bits, sh.forward, deg, fo, mx);
    G2_TRY(cudaMemsetAsync(deg + nv, 0, 8, st));
    G2_TRY(scan(deg, vrp, (uint64_t)nv + 1, &cub_tmp, &cub_cap, st));
    uint64_t m = 0;
    unsigned int max_fwd = 0;
    G2_TRY(cudaMemcpyAsync(&m, vrp + nv, 8, cudaMemcpyDeviceToHost, st));
    G2_TRY(cudaMemcpyAsync(&max_fwd, mx, 4, cudaMemcpyDeviceToHost, st));
    G2_TRY(cudaStreamSynchronize(st));
    g2view::Sizes s;
    s.n = nv;
    s.m = m;
    s.nsrc = nk;
    s.max_fwd = max_fwd;
    const g2view::Layout L(s);
    if (*cap < L.bytes) {
        const uint64_t want = std::max<uint64_t>(L.bytes, *cap + *cap / 2);
        if (*buf) cudaFree(*buf);  // synchronises: the slot's last run has ended anyway
        *buf = nullptr;
        *cap = 0;
        G2_TRY(cudaMalloc(buf, want));
        *cap = want;
    }
    char *b = static_cast<char *>(*buf);
    auto *out_rp = reinterpret_cast<uint64_t *>(b);
    auto *out_fo = reinterpret_cast<uint32_t *>(b + L.fo);
    auto *out_ci = reinterpret_cast<uint32_t *>(b + L.ci);
    auto *out_src = reinterpret_cast<uint32_t *>(b + L.src);
    G2_TRY(cudaMemcpyAsync(out_rp, vrp, 8 * ((uint64_t)nv + 1), cudaMemcpyDeviceToDevice, st));
    if (nv) G2_TRY(cudaMemcpyAsync(out_fo, fo, 4 * (uint64_t)nv, cudaMemcpyDeviceToDevice, st));
    if (nv && m)
        row_write_kernel<<<G, 256, 0, st>>>(hrp, hci, srp, sci, ball, nv, bits, wpre, sh.forward, vrp, out_ci);
    // 5. sources
    if (nk) src_local_kernel<<<G, 256, 0, st>>>(kept, nk, bits, wpre, out_src);
    G2_TRY(cudaGetLastError());
    ctx->launches += 9;
    *out = s;
    return G2_OK;
}

void DeviceViewBuilder::release_host() {
    cudaDeviceSynchronize();  // builds and runs that read the mapped CSR have ended
    for (int k = 0; k < nreg; k++) cudaHostUnregister(reg[k]);
    nreg = 0;
    if (stage_rp) cudaFreeHost(stage_rp);
    if (stage_ci) cudaFreeHost(stage_ci);
    stage_rp = stage_ci = nullptr;
    hrp = nullptr;
    hci = nullptr;
}

DeviceViewBuilder::~DeviceViewBuilder() {
    release_host();
    for (void *p : {(void *)bits, (void *)wcnt, (void *)wpre, (void *)ball, (void *)scalars, (void *)d_roots,
                    (void *)keep, (void *)pos, (void *)kept, (void *)deg, (void *)fo, (void *)vrp, (void *)sstart,
                    (void *)soff, (void *)stage, cub_tmp})
        if (p) cudaFree(p);
}

void view_builder_free(void *builder) { delete static_cast<DeviceViewBuilder *>(builder); }

}  // namespace g2rt

extern "C" int g2_view_materialize_device(g2_ctx *ctx, const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n,
                                          const uint32_t *sources, uint64_t nsrc, uint32_t min_root_degree,
                                          uint32_t flags, g2_view *out) {
    if (!ctx || !row_ptrs || !out || (!sources && nsrc) || (!cols && row_ptrs[n]) || n >= (1ull << 32))
        return G2_ERR_INVALID;
    if (flags & ~(uint32_t)(G2_VIEW_UPPER | G2_VIEW_FORWARD)) return G2_ERR_UNSUPPORTED;
    for (uint64_t i = 0; i < nsrc; i++)
        if (sources[i] >= n) return G2_ERR_INVALID;
    memset(out, 0, sizeof(*out));
    G2_TRY(cudaSetDevice(ctx->device));
    g2view::Shape sh;
    sh.radius = sh.row_radius = 1;
    sh.min_deg = min_root_degree;
    sh.upper = (flags & G2_VIEW_UPPER) != 0;
    sh.forward = (flags & G2_VIEW_FORWARD) != 0;
    // the view lands in the context's first view slot: its graph gives way
    if (ctx->owns_csr) {
        cudaFree(ctx->d_rp);
        cudaFree(ctx->d_ci);
        ctx->rp_cap = ctx->ci_cap = 0;
    }
    ctx->d_rp = nullptr;
    ctx->d_ci = nullptr;
    ctx->owns_csr = false;
    ctx->n = ctx->m = 0;
    g2view::Sizes s;
    uint32_t *ball_host = nullptr;
    {
        if (!ctx->view_builder) ctx->view_builder = new g2rt::DeviceViewBuilder();
        auto &vb = *static_cast<g2rt::DeviceViewBuilder *>(ctx->view_builder);
        int rc = vb.init(ctx, row_ptrs, cols, n, sh);
        if (!rc) rc = vb.build(sources, nsrc, &ctx->view_dev[0], &ctx->view_dev_cap[0], nullptr, &s);
        if (!rc) rc = fail_cuda_if(ctx, cudaStreamSynchronize(nullptr), "view build");
        vb.release_host();  // the build has ended: the host CSR is no longer read
        if (!rc) {
            ball_host = static_cast<uint32_t *>(malloc(4 * std::max<uint64_t>(s.n, 1)));
            if (!ball_host) rc = G2_ERR_OOM;
            else if (s.n) rc = fail_cuda_if(ctx, cudaMemcpy(ball_host, vb.ball, 4 * s.n, cudaMemcpyDeviceToHost),
                                            "view ids");
        }
        if (rc) {
            free(ball_host);
            return rc;
        }
    }
    const g2view::Layout L(s);
    auto *rp = static_cast<uint64_t *>(malloc(8 * (s.n + 1)));
    auto *fo = static_cast<uint32_t *>(malloc(4 * std::max<uint64_t>(s.n, 1)));
    auto *ci = static_cast<uint32_t *>(malloc(4 * std::max<uint64_t>(s.m, 1)));
    auto *src = static_cast<uint32_t *>(malloc(4 * std::max<uint64_t>(s.nsrc, 1)));
    if (!rp || !fo || !ci || !src) {
        free(rp), free(fo), free(ci), free(src), free(ball_host);
        return G2_ERR_OOM;
    }
    const char *b = static_cast<const char *>(ctx->view_dev[0]);
    cudaError_t e = cudaMemcpy(rp, b, 8 * (s.n + 1), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && s.n) e = cudaMemcpy(fo, b + L.fo, 4 * s.n, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && s.m) e = cudaMemcpy(ci, b + L.ci, 4 * s.m, cudaMemcpyDeviceToHost);
    if (e == cudaSuccess && s.nsrc) e = cudaMemcpy(src, b + L.src, 4 * s.nsrc, cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) {
        free(rp), free(fo), free(ci), free(src), free(ball_host);
        return fail_cuda(ctx, e, "view copy-back");
    }
    out->row_ptrs = rp;
    out->cols = ci;
    out->fwd_offsets = fo;
    out->sources = src;
    out->ids = ball_host;
    out->n = s.n;
    out->m = s.m;
    out->nsrc = s.nsrc;
    out->max_fwd = s.max_fwd;
    return G2_OK;
}
