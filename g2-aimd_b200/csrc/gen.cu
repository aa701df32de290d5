// gen.cu - the seeded R-MAT generator on the device.
//
// g2_gen_rmat (csrc/host/graph_host.cpp) builds the benchmark graphs on the
// host; at R-MAT scale 26, edge factor 28 (1.88 G generated edges, 3.6 G
// directed entries after symmetrisation) that takes minutes and ~45 GB of host
// memory.  g2_gen_rmat_device builds the same CSR (same hash per edge, same
// planted cliques, rows sorted and deduplicated) directly into the context:
//   1. degrees: every generated edge (s, d) with s != d adds one to both rows
//      (planted clique edges, made on the host, likewise);
//   2. row starts by an exclusive scan; every edge is generated again and
//      scattered into both rows through per-row atomic cursors;
//   3. rows sorted (segmented sort in calls of <= 2^30 entries, kcore.cu);
//   4. duplicates dropped: kept length per row, a second scan, a compaction.
// Edges are regenerated rather than stored, so the peak is two u32 buffers of
// the undeduplicated directed entries plus the row arrays.  The graph is then
// loaded as by g2_load_csr (owned by the context).
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdint>
#include <vector>

#include "g2_kernels.h"
#include "host/gen_host.h"
#include "runtime_internal.h"

using namespace g2rt;

namespace {

__device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z += 0x9e3779b97f4a7c15ull;
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

struct RmatParams {
    uint64_t seed, seed_mix, ne;
    uint32_t scale, ta, tb, tc;
};

// Edge e of the generator (the host's quadrant walk: four 16-bit draws per word).
__device__ __forceinline__ void rmat_edge(const RmatParams &p, uint64_t e, uint32_t &s, uint32_t &d) {
    s = 0;
    d = 0;
    uint64_t r = 0;
    for (uint32_t l = 0; l < p.scale; l++) {
        if ((l & 3) == 0) r = mix64(p.seed_mix + e * 8 + (l >> 2));
        const uint32_t x = (uint32_t)(r & 0xffff);
        r >>= 16;
        s = (s << 1) | (uint32_t)(x >= p.tb);
        d = (d << 1) | (uint32_t)((x >= p.ta && x < p.tb) || x >= p.tc);
    }
}

__global__ void rmat_degree_kernel(RmatParams p, const uint64_t *extra, uint64_t nextra, unsigned long long *deg) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < p.ne + nextra; e += stride) {
        uint32_t s, d;
        if (e < p.ne) {
            rmat_edge(p, e, s, d);
        } else {
            s = (uint32_t)(extra[e - p.ne] >> 32);
            d = (uint32_t)extra[e - p.ne];
        }
        if (s == d) continue;
        atomicAdd(deg + s, 1ull);
        atomicAdd(deg + d, 1ull);
    }
}

__global__ void rmat_scatter_kernel(RmatParams p, const uint64_t *extra, uint64_t nextra, const uint64_t *start,
                                    unsigned long long *cursor, uint32_t *out) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t e = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; e < p.ne + nextra; e += stride) {
        uint32_t s, d;
        if (e < p.ne) {
            rmat_edge(p, e, s, d);
        } else {
            s = (uint32_t)(extra[e - p.ne] >> 32);
            d = (uint32_t)extra[e - p.ne];
        }
        if (s == d) continue;
        out[start[s] + atomicAdd(cursor + s, 1ull)] = d;
        out[start[d] + atomicAdd(cursor + d, 1ull)] = s;
    }
}

// Kept entries of each sorted row (a warp per row): entries that differ from
// their predecessor.
__global__ void unique_len_kernel(const uint64_t *rp, const uint32_t *ci, uint64_t n, unsigned long long *len) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = w0; v < n; v += nw) {
        const uint64_t lo = rp[v], hi = rp[v + 1];
        unsigned long long c = 0;
        for (uint64_t i = lo + lane; i < hi; i += 32) c += (i == lo || ci[i] != ci[i - 1]);
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) len[v] = c;
    }
}

// Write the kept entries of each row at its new start (a warp per row, ballot
// compaction keeps the order).
__global__ void unique_copy_kernel(const uint64_t *rp, const uint32_t *ci, const uint64_t *nrp, uint64_t n,
                                   uint32_t *out) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = w0; v < n; v += nw) {
        const uint64_t lo = rp[v], hi = rp[v + 1];
        uint64_t o = nrp[v];
        for (uint64_t b = lo; b < hi; b += 32) {
            const uint64_t i = b + lane;
            const bool keep = i < hi && (i == lo || ci[i] != ci[i - 1]);
            const uint32_t m = __ballot_sync(0xffffffffu, keep);
            if (keep) out[o + __popc(m & ((1u << lane) - 1u))] = ci[i];
            o += __popc(m);
        }
    }
}

cudaError_t exclusive_scan(const unsigned long long *in, uint64_t *out, uint64_t items) {
    size_t need = 0;
    const auto *src = reinterpret_cast<const uint64_t *>(in);
    cudaError_t e = cub::DeviceScan::ExclusiveSum(nullptr, need, src, out, (int)items);
    if (e != cudaSuccess) return e;
    void *tmp = nullptr;
    e = cudaMalloc(&tmp, need ? need : 16);
    if (e != cudaSuccess) return e;
    e = cub::DeviceScan::ExclusiveSum(tmp, need, src, out, (int)items);
    cudaError_t f = cudaFree(tmp);
    return e != cudaSuccess ? e : f;
}

}  // namespace

extern "C" int g2_gen_rmat_device(g2_ctx *ctx, uint32_t scale, uint32_t edge_factor, double a, double b, double c,
                                  uint32_t nplanted, uint32_t planted_min, uint32_t planted_max, uint64_t seed,
                                  uint64_t *m_out) {
    if (!ctx || scale < 1 || scale > 30 || edge_factor == 0 || a < 0 || b < 0 || c < 0 || a + b + c > 1)
        return G2_ERR_INVALID;
    const uint64_t n = 1ull << scale;
    std::vector<uint64_t> extra;
    int rc = g2host::planted_edges(n, nplanted, planted_min, planted_max, seed, extra);
    if (rc) return rc;
    G2_TRY(cudaSetDevice(ctx->device));
    RmatParams p;
    p.seed = seed;
    // rnd(seed, stream 2, idx) = mix64(mix64(seed ^ mix64(2 * K)) + idx)
    {
        auto hmix = [](uint64_t z) {
            z += 0x9e3779b97f4a7c15ull;
            z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
            z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
            return z ^ (z >> 31);
        };
        p.seed_mix = hmix(seed ^ hmix(2ull * 0x632be59bd9b4e019ull));
    }
    p.ne = (uint64_t)edge_factor << scale;
    p.scale = scale;
    p.ta = (uint32_t)llround(a * 65536.0);
    p.tb = (uint32_t)llround((a + b) * 65536.0);
    p.tc = (uint32_t)llround((a + b + c) * 65536.0);
    const int G = ctx->sm_count * 8;
    uint64_t *d_extra = nullptr, *start = nullptr, *nrp = nullptr;
    unsigned long long *cnt = nullptr;
    uint32_t *tmp = nullptr, *sorted = nullptr;
    uint64_t m2 = 0, m = 0;
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
        return e == cudaSuccess;
    };
    if (!extra.empty() && (!ok(cudaMalloc(&d_extra, 8 * extra.size())) ||
                           !ok(cudaMemcpy(d_extra, extra.data(), 8 * extra.size(), cudaMemcpyHostToDevice))))
        goto done;
    if (!ok(cudaMalloc(&cnt, 8 * (n + 1))) || !ok(cudaMalloc(&start, 8 * (n + 1))) ||
        !ok(cudaMemset(cnt, 0, 8 * (n + 1))))
        goto done;
    rmat_degree_kernel<<<G, 256>>>(p, d_extra, extra.size(), cnt);
    if (!ok(cudaGetLastError()) || !ok(exclusive_scan(cnt, start, n + 1)) ||
        !ok(cudaMemcpy(&m2, start + n, 8, cudaMemcpyDeviceToHost)))
        goto done;
    if (!ok(cudaMalloc(&tmp, 4 * std::max<uint64_t>(m2, 1))) || !ok(cudaMalloc(&sorted, 4 * std::max<uint64_t>(m2, 1))) ||
        !ok(cudaMemset(cnt, 0, 8 * (n + 1))))
        goto done;
    rmat_scatter_kernel<<<G, 256>>>(p, d_extra, extra.size(), start, cnt, tmp);
    if (!ok(cudaGetLastError())) goto done;
    cudaFree(d_extra);
    d_extra = nullptr;
    if (!ok(g2::sort_rows_device(start, n, m2, tmp, sorted, 1ull << 30, ctx->sm_count))) goto done;
    // deduplicate: kept length per row (into cnt), row pointers, compaction into tmp
    unique_len_kernel<<<G, 256>>>(start, sorted, n, cnt);
    if (!ok(cudaGetLastError()) || !ok(cudaMalloc(&nrp, 8 * (n + 1))) || !ok(cudaMemset(cnt + n, 0, 8)) ||
        !ok(exclusive_scan(cnt, nrp, n + 1)) || !ok(cudaMemcpy(&m, nrp + n, 8, cudaMemcpyDeviceToHost)))
        goto done;
    unique_copy_kernel<<<G, 256>>>(start, sorted, nrp, n, tmp);
    if (!ok(cudaGetLastError()) || !ok(cudaDeviceSynchronize())) goto done;
done:
    cudaFree(d_extra);
    cudaFree(cnt);
    cudaFree(start);
    cudaFree(sorted);
    if (e != cudaSuccess) {
        cudaFree(tmp);
        cudaFree(nrp);
        return e == cudaErrorNotSupported ? G2_ERR_UNSUPPORTED
               : e == cudaErrorMemoryAllocation ? (cudaGetLastError(), G2_ERR_OOM)
                                                : fail_cuda(ctx, e, "g2_gen_rmat_device");
    }
    // the generated CSR becomes the context's graph (tmp holds m entries of its
    // m2-entry allocation)
    if (ctx->owns_csr) {
        cudaFree(ctx->d_rp);
        cudaFree(ctx->d_ci);
    }
    ctx->d_rp = nrp;
    ctx->d_ci = tmp;
    ctx->owns_csr = true;
    ctx->rp_cap = n + 1;
    ctx->ci_cap = std::max<uint64_t>(m2, 1);
    ctx->n = n;
    ctx->m = m;
    if (m_out) *m_out = m;
    return g2_after_load(ctx);
}
