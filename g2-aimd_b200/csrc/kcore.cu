// kcore.cu - degeneracy order of the loaded graph on the device, and the
// recode that renames vertices by it.
//
// Replaces the host preprocessing of kmeans/kcore.cpp:39-191 (k-core peeling,
// then a degree sort inside each shell and a recode): core numbers by
// level-synchronous peeling (every vertex of remaining degree <= k leaves in
// rounds, its live neighbours lose one degree each; core numbers are unique, so
// any peeling order gives the same ones), then the order (core, degree, id)
// ascending by a stable radix sort of (core << 32 | degree) over ids.  The
// result equals g2_degeneracy_order's (csrc/host/graph_host.cpp) exactly.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cstdint>
#include <vector>

#include "g2_kernels.h"

namespace g2 {

namespace {

// Vertices still alive with degree <= k leave: core = k, appended to the frontier.
__global__ void peel_select_kernel(const uint32_t *deg, uint8_t *alive, uint32_t *core, uint64_t n, uint32_t k,
                                   uint32_t *frontier, unsigned long long *nfront) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
        if (alive[v] && deg[v] <= k) {
            alive[v] = 0;
            core[v] = k;
            frontier[atomicAdd(nfront, 1ull)] = (uint32_t)v;
        }
    }
}

// Live neighbours of the frontier lose one degree per frontier neighbour (a
// warp per frontier vertex); the smallest live degree is collected for the
// next level.
__global__ void peel_update_kernel(const uint64_t *rp, const uint32_t *ci, const uint32_t *frontier,
                                   const unsigned long long *nfront, const uint8_t *alive, uint32_t *deg) {
    const uint64_t nf = *nfront;
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = w0; i < nf; i += nw) {
        const uint32_t v = frontier[i];
        for (uint64_t e = rp[v] + lane; e < rp[v + 1]; e += 32) {
            const uint32_t u = ci[e];
            if (alive[u]) atomicSub(deg + u, 1u);
        }
    }
}

__global__ void min_alive_degree_kernel(const uint32_t *deg, const uint8_t *alive, uint64_t n, unsigned int *out) {
    unsigned int m = 0xffffffffu;
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        if (alive[v] && deg[v] < m) m = deg[v];
    for (int o = 16; o > 0; o >>= 1) {
        const unsigned int y = __shfl_xor_sync(0xffffffffu, m, o);
        m = y < m ? y : m;
    }
    if ((threadIdx.x & 31u) == 0 && m != 0xffffffffu) atomicMin(out, m);
}

__global__ void init_kernel(const uint64_t *rp, uint64_t n, uint32_t *deg, uint8_t *alive,
                            unsigned long long *keys, uint32_t *ids) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
        deg[v] = (uint32_t)(rp[v + 1] - rp[v]);
        alive[v] = 1;
        ids[v] = (uint32_t)v;
        keys[v] = 0;
    }
}

__global__ void order_keys_kernel(const uint64_t *rp, const uint32_t *core, uint64_t n, unsigned long long *keys) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        keys[v] = ((unsigned long long)core[v] << 32) | (unsigned long long)(rp[v + 1] - rp[v]);
}

__global__ void scatter_perm_kernel(const uint32_t *ord, uint64_t n, uint32_t *perm) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        perm[ord[i]] = (uint32_t)i;
}

// Row length of each vertex under its new name (entry n stays 0 for the scan).
__global__ void recode_degrees_kernel(const uint64_t *rp, const uint32_t *perm, uint64_t n, uint64_t *deg) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x)
        deg[perm[v]] = rp[v + 1] - rp[v];
}

// Row of v, renamed, written unsorted at its new place (a warp per row).
__global__ void recode_scatter_kernel(const uint64_t *rp, const uint32_t *ci, const uint32_t *perm,
                                      const uint64_t *new_rp, uint64_t n, uint32_t *out) {
    const uint32_t lane = threadIdx.x & 31u;
    const uint64_t w0 = ((uint64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t v = w0; v < n; v += nw) {
        const uint64_t lo = rp[v], len = rp[v + 1] - lo, base = new_rp[perm[v]];
        for (uint64_t i = lane; i < len; i += 32) out[base + i] = perm[ci[lo + i]];
    }
}

// Offsets of rows [r0, r0 + rows] relative to row r0 (segmented sort of one chunk).
__global__ void chunk_offsets_kernel(const uint64_t *new_rp, uint64_t r0, uint64_t rows, int *off) {
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i <= rows; i += (uint64_t)gridDim.x * blockDim.x)
        off[i] = (int)(new_rp[r0 + i] - new_rp[r0]);
}

}  // namespace

// Sort every row of a CSR whose row pointers (device, n+1) are rp: the rows of
// `in` are sorted into `out`, in CUB segmented-sort calls of at most max_chunk
// entries (CUB counts items and segments in int).  A row longer than max_chunk:
// cudaErrorNotSupported.  Synchronous.
cudaError_t sort_rows_device(const uint64_t *rp, uint64_t n, uint64_t m, const uint32_t *in, uint32_t *out,
                             uint64_t max_chunk, int sms) {
    max_chunk = std::min<uint64_t>(std::max<uint64_t>(max_chunk, 1), (uint64_t)INT_MAX);
    int *off = nullptr;
    void *cub_tmp = nullptr;
    size_t cub_bytes = 0, need = 0;
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
        return e == cudaSuccess;
    };
    const int G = sms * 8;
    uint32_t *tmp = const_cast<uint32_t *>(in);
    const uint64_t *nrp = rp;
    std::vector<uint64_t> cuts;  // row boundaries of the sort calls
    if (m <= max_chunk) {
        cuts = {0, n};
    } else {
        std::vector<uint64_t> h(n + 1);
        if (!ok(cudaMemcpy(h.data(), nrp, 8 * (n + 1), cudaMemcpyDeviceToHost))) goto done;
        cuts.push_back(0);
        uint64_t r = 0;
        while (r < n) {
            if (h[r + 1] - h[r] > max_chunk) {
                e = cudaErrorNotSupported;
                goto done;
            }
            // the last row r1 with h[r1] - h[r] <= max_chunk
            const uint64_t r1 =
                (uint64_t)(std::upper_bound(h.begin() + r, h.end(), h[r] + max_chunk) - h.begin()) - 1;
            r = std::min<uint64_t>(r1, n);
            cuts.push_back(r);
        }
    }
    if (!ok(cudaMalloc(&off, sizeof(int) * (std::min<uint64_t>(n, max_chunk) + 2)))) goto done;
    for (size_t k = 0; k + 1 < cuts.size(); k++) {
        const uint64_t r0 = cuts[k], rows = cuts[k + 1] - r0;
        if (!rows) continue;
        uint64_t base = 0, items = 0;
        if (!ok(cudaMemcpy(&base, nrp + r0, 8, cudaMemcpyDeviceToHost)) ||
            !ok(cudaMemcpy(&items, nrp + r0 + rows, 8, cudaMemcpyDeviceToHost)))
            goto done;
        items -= base;
        if (!items) continue;
        if (rows + 1 > (uint64_t)INT_MAX) {
            e = cudaErrorNotSupported;
            goto done;
        }
        if (rows + 2 > std::min<uint64_t>(n, max_chunk) + 2) {  // more rows than the offsets buffer holds
            cudaFree(off);
            off = nullptr;
            if (!ok(cudaMalloc(&off, sizeof(int) * (rows + 1)))) goto done;
        }
        chunk_offsets_kernel<<<G, 256>>>(nrp, r0, rows, off);
        need = 0;
        if (!ok(cub::DeviceSegmentedSort::SortKeys(nullptr, need, tmp + base, out + base, (int)items, (int)rows, off,
                                                    off + 1)))
            goto done;
        if (need > cub_bytes) {
            cudaFree(cub_tmp);
            cub_tmp = nullptr;
            cub_bytes = need;
            if (!ok(cudaMalloc(&cub_tmp, cub_bytes))) goto done;
        }
        if (!ok(cub::DeviceSegmentedSort::SortKeys(cub_tmp, need, tmp + base, out + base, (int)items, (int)rows, off,
                                                    off + 1)))
            goto done;
    }
    ok(cudaGetLastError());
    ok(cudaDeviceSynchronize());
done:
    cudaFree(off);
    cudaFree(cub_tmp);
    return e;
}

cudaError_t recode_device(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint64_t m, const uint32_t *perm,
                          uint64_t max_chunk, int sms, uint64_t **new_rp, uint32_t **new_ci) {
    *new_rp = nullptr;
    *new_ci = nullptr;
    if (n + 1 > (uint64_t)INT_MAX) return cudaErrorNotSupported;  // the scan counts items in int
    max_chunk = std::min<uint64_t>(std::max<uint64_t>(max_chunk, 1), (uint64_t)INT_MAX);
    uint64_t *nrp = nullptr, *deg = nullptr;
    uint32_t *tmp = nullptr, *nci = nullptr;
    void *cub_tmp = nullptr;
    size_t cub_bytes = 0, need = 0;
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
        return e == cudaSuccess;
    };
    const int G = sms * 8;
    if (!ok(cudaMalloc(&nrp, 8 * (n + 1))) || !ok(cudaMalloc(&deg, 8 * (n + 1))) ||
        !ok(cudaMalloc(&tmp, 4 * std::max<uint64_t>(m, 1))) || !ok(cudaMalloc(&nci, 4 * std::max<uint64_t>(m, 1))) ||
        !ok(cudaMemset(deg, 0, 8 * (n + 1))))
        goto done;
    recode_degrees_kernel<<<G, 256>>>(rp, perm, n, deg);
    // exclusive scan: row pointers of the renamed rows (entry n = m)
    if (!ok(cub::DeviceScan::ExclusiveSum(nullptr, need, deg, nrp, (int)(n + 1)))) goto done;
    cub_bytes = need;
    if (!ok(cudaMalloc(&cub_tmp, cub_bytes ? cub_bytes : 16)) ||
        !ok(cub::DeviceScan::ExclusiveSum(cub_tmp, need, deg, nrp, (int)(n + 1))))
        goto done;
    recode_scatter_kernel<<<G, 256>>>(rp, ci, perm, nrp, n, tmp);
    if (!ok(cudaGetLastError())) goto done;
    // sort the rows, in calls of at most max_chunk entries
    if (!ok(sort_rows_device(nrp, n, m, tmp, nci, max_chunk, sms))) goto done;
    ok(cudaGetLastError());
    ok(cudaDeviceSynchronize());
done:
    cudaFree(deg);
    cudaFree(tmp);
    cudaFree(cub_tmp);
    if (e != cudaSuccess) {
        cudaFree(nrp);
        cudaFree(nci);
        return e;
    }
    *new_rp = nrp;
    *new_ci = nci;
    return cudaSuccess;
}

// perm (new id of each vertex) and core numbers of the CSR (rp, ci) with n
// vertices; device buffers.  Synchronous (the level loop reads counts back).
cudaError_t degeneracy_order_device(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint32_t *perm,
                                    uint32_t *core, int sms, uint64_t *rounds) {
    *rounds = 0;
    if (n == 0) return cudaSuccess;
    uint32_t *deg = nullptr, *frontier = nullptr, *ids = nullptr, *ids2 = nullptr;
    uint8_t *alive = nullptr;
    unsigned long long *keys = nullptr, *keys2 = nullptr, *nfront = nullptr;
    unsigned int *dmin = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
        return e == cudaSuccess;
    };
    const int G = sms * 8;
    if (!ok(cudaMalloc(&deg, n * 4)) || !ok(cudaMalloc(&frontier, n * 4)) || !ok(cudaMalloc(&ids, n * 4)) ||
        !ok(cudaMalloc(&ids2, n * 4)) || !ok(cudaMalloc(&alive, n)) || !ok(cudaMalloc(&keys, n * 8)) ||
        !ok(cudaMalloc(&keys2, n * 8)) || !ok(cudaMalloc(&nfront, 8)) || !ok(cudaMalloc(&dmin, 4)))
        goto done;
    init_kernel<<<G, 256>>>(rp, n, deg, alive, keys, ids);
    {
        uint64_t removed = 0;
        uint32_t k = 0;
        while (removed < n) {
            // next level: the smallest live degree, if above the current one
            if (!ok(cudaMemset(dmin, 0xff, 4))) goto done;
            min_alive_degree_kernel<<<G, 256>>>(deg, alive, n, dmin);
            unsigned int m = 0;
            if (!ok(cudaMemcpy(&m, dmin, 4, cudaMemcpyDeviceToHost))) goto done;
            if (m > k) k = m;
            // peel rounds at level k until no live vertex has degree <= k
            for (;;) {
                if (!ok(cudaMemset(nfront, 0, 8))) goto done;
                peel_select_kernel<<<G, 256>>>(deg, alive, core, n, k, frontier, nfront);
                unsigned long long nf = 0;
                if (!ok(cudaMemcpy(&nf, nfront, 8, cudaMemcpyDeviceToHost))) goto done;
                ++*rounds;
                if (nf == 0) break;
                removed += nf;
                peel_update_kernel<<<G, 256>>>(rp, ci, frontier, nfront, alive, deg);
            }
            k++;
        }
    }
    order_keys_kernel<<<G, 256>>>(rp, core, n, keys);
    if (!ok(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, keys, keys2, ids, ids2, (int)n)) ||
        !ok(cudaMalloc(&tmp, tmp_bytes ? tmp_bytes : 16)) ||
        !ok(cub::DeviceRadixSort::SortPairs(tmp, tmp_bytes, keys, keys2, ids, ids2, (int)n)))
        goto done;
    scatter_perm_kernel<<<G, 256>>>(ids2, n, perm);
    ok(cudaGetLastError());
    ok(cudaDeviceSynchronize());
done:
    cudaFree(deg);
    cudaFree(frontier);
    cudaFree(ids);
    cudaFree(ids2);
    cudaFree(alive);
    cudaFree(keys);
    cudaFree(keys2);
    cudaFree(nfront);
    cudaFree(dmin);
    cudaFree(tmp);
    return e;
}

}  // namespace g2
