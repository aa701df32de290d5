// g2_handoff.cuh - the record queue through which walks hand work to idle warps.
//
// Used by the persistent MCE and GMatch kernels.  A walk that runs long while
// other warps are idle writes some of its pending work as records; idle warps
// take tickets (the index of the next record, reserved or not yet) and run the
// record of their ticket once it is published.  Args is MceArgs or MatchArgs:
//   records/rec_stride/rec_cap  the record slots
//   ready[i]                    epoch of the run that published slot i
//   nrec                        slots reserved so far (one atomic per reservation)
//   qctl[kQHead]                tickets taken
//   qctl[kQOut]                 outstanding work: warps holding queue tasks plus
//                               reserved, unfinished records.  It is raised before
//                               work is published and lowered when it is done, by
//                               warps that are themselves counted, so once it reads
//                               zero no record can appear any more.
// Every wait is bounded (wait_cycles); a warp that gives up flags kStatusWaitLimit.
#pragma once

#include <cstdint>

#include "g2_device.cuh"
#include "g2_kernels.h"

namespace g2 {

__device__ __forceinline__ unsigned long long vload(const unsigned long long *p) {
    return *reinterpret_cast<const volatile unsigned long long *>(p);
}
__device__ __forceinline__ uint32_t vload32(const uint32_t *p) { return *reinterpret_cast<const volatile uint32_t *>(p); }

// Reserve n consecutive records with one atomic (no retries: many warps hand
// off work at the same moment).  The slots that exist are added to the
// outstanding count before any of them is published (the caller is itself
// outstanding, so the count cannot touch zero meanwhile).  If the slots run
// past the end of the buffer the ones below the end are published as void
// (word 1 = kVoidRecord; their ticket holders skip them) and ~0 is returned.
template <class Args>
__device__ __forceinline__ unsigned long long reserve_records(const Args &a, uint32_t n) {
    unsigned long long base = 0;
    if (lane_id() == 0) {
        base = atomicAdd(a.nrec, (unsigned long long)n);
        const unsigned long long end = base + n < a.rec_cap ? base + n : a.rec_cap;
        if (end > base) atomicAdd(a.qctl + kQOut, end - base);
    }
    base = __shfl_sync(G2_FULL, base, 0);
    if (base + n <= a.rec_cap) return base;
    for (unsigned long long i = base + lane_id(); i < a.rec_cap && i < base + n; i += 32)
        a.records[i * a.rec_stride + 1] = kVoidRecord;
    __syncwarp();
    __threadfence();
    for (unsigned long long i = base + lane_id(); i < a.rec_cap && i < base + n; i += 32)
        *reinterpret_cast<volatile uint32_t *>(a.ready + i) = a.epoch;
    __syncwarp();
    return ~0ull;
}

// Make records [k0, k1) visible to their ticket holders: data first, then the
// ready words.
template <class Args>
__device__ __forceinline__ void publish_records(const Args &a, unsigned long long k0, unsigned long long k1) {
    __syncwarp();
    __threadfence();
    for (unsigned long long i = k0 + lane_id(); i < k1; i += 32)
        *reinterpret_cast<volatile uint32_t *>(a.ready + i) = a.epoch;
    __syncwarp();
}

// Do idle warps hold tickets past the last reserved record?  (lane 0's read,
// broadcast to the warp)
template <class Args>
__device__ __forceinline__ bool handoff_wanted(const Args &a) {
    int want = 0;
    if (lane_id() == 0) want = vload(a.qctl + kQHead) > vload(a.nrec);
    return __shfl_sync(G2_FULL, want, 0) != 0;
}

// A warp counts itself before taking queue tasks (and uncounts after).
template <class Args>
__device__ __forceinline__ void outstanding_add(const Args &a, bool on, long long d) {
    if (on && lane_id() == 0) {
        atomicAdd(a.qctl + kQOut, (unsigned long long)d);
        if (d > 0) __threadfence();  // counted before the task is taken
    }
}

// Phase 2 of a pass that hands off work: take tickets and run their records
// (run(h) runs record h) until no work is outstanding.
// Backoff cap of a waiting warp.  Thousands of waiting warps poll; with a 2 us
// cap their traffic on the counters' L2 slice slowed the warps still working
// (plan walks on R-MAT s16: 8.7 s -> 6.6 s with 16 us), with no loss for MCE.
constexpr uint32_t kMaxSleepNs = 16384;

template <class Args, class Run>
__device__ void run_record_queue(const Args &a, Run run) {
    const uint32_t lane = lane_id();
    unsigned long long h = 0;
    if (lane == 0) h = atomicAdd(a.qctl + kQHead, 1ull);
    h = __shfl_sync(G2_FULL, h, 0);
    uint32_t sleep_ns = 32, polls = 0;
    long long w0 = clock64();
    for (;;) {
        int action = 0;  // 0 wait, 1 run record h, 2 leave
        if (lane == 0) {
            if (h < a.rec_cap && vload32(a.ready + h) == a.epoch) {
                action = 1;
            } else if ((++polls & 3u) == 0) {  // the shared counter on every 4th poll only
                __threadfence();  // whatever this warp saw taken was counted first
                if (vload(a.qctl + kQOut) == 0) action = 2;
            }
        }
        action = __shfl_sync(G2_FULL, action, 0);
        if (action == 1) {
            __threadfence();
            run(h);
            if (lane == 0) {
                atomicAdd(a.qctl + kQOut, ~0ull);  // -1
                h = atomicAdd(a.qctl + kQHead, 1ull);
            }
            h = __shfl_sync(G2_FULL, h, 0);
            sleep_ns = 32;
            w0 = clock64();
            continue;
        }
        if (action == 2) break;
        if (clock64() - w0 > (long long)a.wait_cycles) {
            if (lane == 0) atomicOr(a.status, kStatusWaitLimit);
            break;
        }
        __nanosleep(sleep_ns);
        sleep_ns = sleep_ns < kMaxSleepNs ? sleep_ns * 2 : kMaxSleepNs;
    }
}

}  // namespace g2
