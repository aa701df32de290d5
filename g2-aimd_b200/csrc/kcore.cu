// kcore.cu - degeneracy order of the loaded graph on the device.
//
// Replaces the host preprocessing of kmeans/kcore.cpp:39-191 (k-core peeling,
// then a degree sort inside each shell and a recode): core numbers by
// level-synchronous peeling (every vertex of remaining degree <= k leaves in
// rounds, its live neighbours lose one degree each; core numbers are unique, so
// any peeling order gives the same ones), then the order (core, degree, id)
// ascending by a stable radix sort of (core << 32 | degree) over ids.  The
// result equals g2_degeneracy_order's (csrc/host/graph_host.cpp) exactly.
#include <cub/cub.cuh>

#include <cstdint>

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

}  // namespace

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
