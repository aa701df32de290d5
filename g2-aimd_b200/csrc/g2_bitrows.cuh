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

// Row of u against P0 = ci[split, split+p), all lanes participate; rowbuf is this
// warp's shared scratch of 32*WPL words.
template <int WPL>
__device__ void build_row(const uint64_t *rp, const uint32_t *ci, uint32_t v, uint64_t split, uint32_t p,
                          uint32_t W, uint32_t pmax, uint32_t u, Row<WPL> &row, uint32_t *rowbuf) {
    const uint32_t lane = lane_id();
    const uint64_t ulo = ldg(rp + u), uhi = ldg(rp + u + 1);
    const uint64_t du = uhi - ulo;
    row_zero(row);
    if (du == 0) return;
    if ((uint64_t)p * ilog2p1(du) <= du * ilog2p1(p)) {
        // test every P0 member in N(u)
        for (uint32_t c = 0; c < W; c++) {
            uint32_t j = 32u * c + lane;
            bool f = j < p && contains(ci, ulo, uhi, ldg(ci + split + j));
            uint32_t bits = __ballot_sync(G2_FULL, f);
#pragma unroll
            for (int s = 0; s < WPL; s++)
                if ((c >> 5) == (uint32_t)s && lane == (c & 31u)) row.w[s] = bits;
        }
    } else {
        // locate every neighbour of u inside P0
#pragma unroll
        for (int s = 0; s < WPL; s++)
            if (lane + 32u * s < W) rowbuf[lane + 32u * s] = 0u;
        __syncwarp();
        for (uint64_t e = ulo + lane; e < uhi; e += 32) {
            uint32_t y = ldg(ci + e);
            if (y > v && y <= pmax) {
                uint64_t j = lower_bound(ci, split, split + p, y);
                if (j < split + p && ldg(ci + j) == y) {
                    uint32_t jj = (uint32_t)(j - split);
                    atomicOr(rowbuf + (jj >> 5), 1u << (jj & 31u));
                }
            }
        }
        __syncwarp();
#pragma unroll
        for (int s = 0; s < WPL; s++) row.w[s] = (lane + 32u * s < W) ? rowbuf[lane + 32u * s] : 0u;
        __syncwarp();
    }
}

}  // namespace g2
