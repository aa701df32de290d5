// g2_device.cuh - warp-level primitives shared by the enumeration kernels.
//
// All kernels here are integer/HBM-bound: no tensor cores.  A warp owns one
// task at a time; lists are sorted uint32 vertex ids; bitmaps over a root's
// local vertex set are distributed across the warp (word w lives in lane
// w % 32, register slot w / 32).
#pragma once

#include <cstdint>

#define G2_FULL 0xffffffffu

namespace g2 {

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Read-only, L1-cacheable load (graph arrays never change during a kernel).
__device__ __forceinline__ uint32_t ldg(const uint32_t *p) { return __ldg(p); }
__device__ __forceinline__ uint64_t ldg(const uint64_t *p) { return __ldg(reinterpret_cast<const unsigned long long *>(p)); }

// First index in [lo, hi) with a[i] >= key (one lane).
__device__ __forceinline__ uint64_t lower_bound(const uint32_t *a, uint64_t lo, uint64_t hi, uint32_t key) {
    while (lo < hi) {
        uint64_t mid = lo + ((hi - lo) >> 1);
        if (ldg(a + mid) < key) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

__device__ __forceinline__ bool contains(const uint32_t *a, uint64_t lo, uint64_t hi, uint32_t key) {
    uint64_t i = lower_bound(a, lo, hi, key);
    return i < hi && ldg(a + i) == key;
}

// Exclusive prefix of `pred` over the warp and the warp total.
__device__ __forceinline__ uint32_t warp_scan(bool pred, uint32_t &total) {
    uint32_t b = __ballot_sync(G2_FULL, pred);
    total = __popc(b);
    return __popc(b & ((1u << lane_id()) - 1u));
}

__device__ __forceinline__ unsigned long long warp_max_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        unsigned long long w = __shfl_xor_sync(G2_FULL, v, o);
        v = w > v ? w : v;
    }
    return v;
}

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(G2_FULL, v, o);
    return v;
}

// Lane 0 grabs `chunk` tasks from a global counter; all lanes get the start.
__device__ __forceinline__ unsigned long long grab(unsigned long long *head, uint32_t chunk) {
    unsigned long long t = 0;
    if (lane_id() == 0) t = atomicAdd(head, (unsigned long long)chunk);
    return __shfl_sync(G2_FULL, t, 0);
}

}  // namespace g2
