// noalloc.cu - a plan-driven count that allocates no memory.
//
// g2_match_run / g2_match_run_device keep their scratch (the per-warp DFS slabs,
// the forward-list offsets, the task list, the queue counters) in buffers that
// the context allocates with cudaMalloc.  Some callers cannot let a library do
// that: an application whose device memory is owned by its own caching
// allocator or by a fixed budget (a cudaMalloc from the library would bypass
// that accounting and can fail or fragment the pool under memory pressure), and
// code on a latency-critical path, where cudaMalloc / cudaFree may synchronise
// the device.  For them, g2_match_count_noalloc runs the same match kernel with
// its scratch in the file-scope device array below, which every GPU that loads
// this library holds from module load until process exit.
//
// Limits and sharing (also stated in include/g2_aimd.h):
//   * scratch size G2_NOALLOC_SCRATCH_BYTES (32 MiB); graphs with more than
//     G2_NOALLOC_MAX_VERTICES vertices are rejected with G2_ERR_UNSUPPORTED;
//   * the array is shared by every call on a device and keeps the contents of
//     the last call; the queue counter, the status word and the caller's count
//     are cleared at the start of each call, everything else is rewritten before
//     it is read;
//   * two calls whose work overlaps on the GPU (different streams, or different
//     host threads on one device) race on that array and give wrong counts:
//     serialise them.  The plan travels as a kernel argument, so a call may
//     overlap context runs (g2_match_run*) of any plan;
//   * every call looks up the array's device address on the current device
//     (cudaGetSymbolAddress allocates nothing), so a context that was torn
//     down and created again never sees a stale address;
//   * a device-side failure (the kernel's status word non-zero, e.g. a
//     candidate stack too small for the query) is reported on the stream:
//     *d_count is set to G2_NOALLOC_FAILED (UINT64_MAX) instead of a count.
#include <cuda_runtime.h>

#include <cstring>

#include "g2_aimd.h"
#include "g2_kernels.h"

namespace {

constexpr uint64_t kWords = G2_NOALLOC_SCRATCH_BYTES / sizeof(uint32_t);
constexpr uint64_t kHeadWords = 64;  // [0..1] queue head (u64), [2] status word
constexpr int kWarpsPerBlock = 4;

static __device__ __align__(256) uint32_t g_noalloc_scratch[kWords];

// The array's address on the current device.  In host code the symbol itself
// is only a host-side stand-in; kernels must be given this address.
int scratch_address(uint32_t **out) {
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) return G2_ERR_CUDA;
    *out = static_cast<uint32_t *>(p);
    return G2_OK;
}

// Runs after the count on the same stream: a non-zero status word replaces the
// count by the failure sentinel.
__global__ void noalloc_status_kernel(const int *status, unsigned long long *count) {
    if (*status != 0) *count = G2_NOALLOC_FAILED;
}

// fo[v] (offset of the first neighbour larger than v) and the identity task list.
__global__ void noalloc_prepare_kernel(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint32_t *fo,
                                       uint32_t *tasks) {
    for (uint64_t v = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; v < n; v += (uint64_t)gridDim.x * blockDim.x) {
        uint64_t lo = rp[v], hi = rp[v + 1], a = lo, b = hi;
        while (a < b) {
            uint64_t mid = a + ((b - a) >> 1);
            if (ci[mid] <= (uint32_t)v) a = mid + 1;
            else b = mid;
        }
        fo[v] = (uint32_t)(a - lo);
        tasks[v] = (uint32_t)v;
    }
}

// g2_plan (reference indexing) -> device plan (everything by position).
int to_dev_plan(const g2_plan *p, g2::DevPlan *d, bool *clique) {
    const uint32_t k = p->k;
    if (k < 2 || k > G2_MAX_QUERY) return G2_ERR_UNSUPPORTED;
    memset(d, 0, sizeof(*d));
    d->k = k;
    for (uint32_t u = 0; u < k; u++)
        if (p->order[u] >= k || p->id2order[p->order[u]] != u) return G2_ERR_INVALID;
    bool cl = true;
    for (uint32_t i = 0; i < k; i++) {
        const uint32_t u = p->order[i];
        if (i > 0 && (p->bn_count[i] == 0 || p->bn_count[i] > k)) return G2_ERR_INVALID;
        if (p->cond_count[u] > k) return G2_ERR_INVALID;
        d->bn_count[i] = p->bn_count[i];
        for (uint32_t j = 0; j < p->bn_count[i]; j++) {
            if (p->bn[i][j] >= k) return G2_ERR_INVALID;
            const uint32_t pos = p->id2order[p->bn[i][j]];
            if (pos >= i) return G2_ERR_INVALID;
            d->bn_pos[i][j] = pos;
        }
        d->cond_count[i] = p->cond_count[u];
        uint32_t larger = 0;
        for (uint32_t j = 0; j < p->cond_count[u]; j++) {
            if (p->cond[u][j][1] >= k || p->cond[u][j][0] > G2_COND_NON_EQUAL) return G2_ERR_INVALID;
            const uint32_t pos = p->id2order[p->cond[u][j][1]];
            if (pos >= i) return G2_ERR_INVALID;
            d->cond_op[i][j] = p->cond[u][j][0];
            d->cond_pos[i][j] = pos;
            larger += p->cond[u][j][0] == G2_COND_LARGER_THAN;
        }
        if (i > 0 && (p->bn_count[i] != i || larger != i)) cl = false;
        d->share[i] = p->share[i];
    }
    d->clique = cl ? 1u : 0u;
    *clique = cl;
    return G2_OK;
}

}  // namespace

extern "C" int g2_match_count_noalloc(const uint64_t *d_row_ptrs, const uint32_t *d_cols, uint64_t n, uint64_t m,
                                      const g2_plan *plan, uint64_t *d_count, void *stream) {
    if (!d_row_ptrs || (!d_cols && m) || !plan || !d_count) return G2_ERR_INVALID;
    if (n > G2_NOALLOC_MAX_VERTICES) return G2_ERR_UNSUPPORTED;
    g2::DevPlan dp;
    bool clique = false;
    int rc = to_dev_plan(plan, &dp, &clique);
    if (rc) return rc;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return G2_ERR_CUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return G2_ERR_CUDA;
    uint32_t *S = nullptr;
    rc = scratch_address(&S);
    if (rc) return rc;
    // layout: [head/status kHeadWords] [fo n] [tasks n] [per-warp slabs]
    uint32_t *fo = S + kHeadWords;
    uint32_t *tasks = fo + n;
    const uint64_t slab0 = (kHeadWords + 2 * n + 63) & ~63ull;
    const int blocks = sms, wpb = kWarpsPerBlock;
    const uint64_t nwarps = (uint64_t)blocks * wpb;
    if (slab0 >= kWords) return G2_ERR_UNSUPPORTED;
    const uint64_t wpw = ((kWords - slab0) / nwarps) & ~63ull;
    if (wpw / (dp.k > 2 ? dp.k - 2 : 1) < 64) return G2_ERR_UNSUPPORTED;  // slabs too small for this query
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // what must start at zero: the queue head, the status word, the count
    if (cudaMemsetAsync(S, 0, kHeadWords * sizeof(uint32_t), st) != cudaSuccess) return G2_ERR_CUDA;
    if (cudaMemsetAsync(d_count, 0, sizeof(uint64_t), st) != cudaSuccess) return G2_ERR_CUDA;
    if (n) noalloc_prepare_kernel<<<sms * 4, 256, 0, st>>>(d_row_ptrs, d_cols, n, fo, tasks);
    if (cudaGetLastError() != cudaSuccess) return G2_ERR_CUDA;
    g2::MatchArgs a{};
    a.rp = d_row_ptrs;
    a.ci = d_cols;
    a.fo = fo;
    a.tasks = tasks;
    a.ntasks = n;
    a.head = reinterpret_cast<unsigned long long *>(S);
    a.chunk = 4;
    a.scratch = S + slab0;
    a.words_per_warp = wpw;
    a.out = reinterpret_cast<unsigned long long *>(d_count);
    a.status = reinterpret_cast<int *>(S + 2);
    a.p0_words = g2::match_p0_words(1, clique, dp.k, false);
    if (g2::match_launch(dp, a, blocks, wpb, st, clique, 1, 0) != cudaSuccess) return G2_ERR_CUDA;
    noalloc_status_kernel<<<1, 1, 0, st>>>(a.status, a.out);
    if (cudaGetLastError() != cudaSuccess) return G2_ERR_CUDA;
    return G2_OK;
}
