// view_device.h - radius-1 views of a host CSR built on the device
// (view_device.cu; internal to libg2aimd.so).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "host/view_host.h"

struct g2_ctx;

namespace g2rt {

// Builds the views of a view run on the GPU from the host CSR, read through
// mapped pinned memory.  Same output as g2view::Builder::fill_packed for shapes
// with radius 1, row radius 1 and no ego rows.
struct DeviceViewBuilder {
    // Map the host CSR for the device (pinned memory in place, else registered
    // for the call, else copied to mapped staging buffers) and allocate the
    // n-sized work arrays.
    int init(g2_ctx *ctx, const uint64_t *host_rp, const uint32_t *host_ci, uint64_t n, const g2view::Shape &shape);
    // Undo init's host mapping (registrations, staging copies); the device
    // work arrays stay for the next call.
    void release_host();
    // The view of `roots` (host array) into *buf (a device slot, grown to fit),
    // enqueued on st; returns once its sizes are known (the writes may still be
    // in flight on st).
    int build(const uint32_t *roots, uint64_t nroots, void **buf, uint64_t *cap, cudaStream_t st,
              g2view::Sizes *out);
    ~DeviceViewBuilder();

    g2_ctx *ctx = nullptr;
    uint64_t n = 0, words = 0;
    g2view::Shape sh;
    const uint64_t *hrp = nullptr;  // device-side pointers to the host CSR
    const uint32_t *hci = nullptr;
    void *reg[2] = {nullptr, nullptr};  // page ranges registered for the call
    int nreg = 0;
    void *stage_rp = nullptr, *stage_ci = nullptr;  // mapped copies if registering failed
    uint64_t n_cap = 0;  // graph size the n-sized arrays were allocated for
    uint32_t *bits = nullptr, *wcnt = nullptr, *wpre = nullptr, *ball = nullptr;
    unsigned long long *scalars = nullptr;
    uint32_t *d_roots = nullptr, *keep = nullptr, *pos = nullptr, *kept = nullptr;
    uint64_t roots_cap = 0;
    unsigned long long *deg = nullptr;
    uint32_t *fo = nullptr;
    uint64_t *vrp = nullptr;
    uint64_t *sstart = nullptr, *soff = nullptr;  // staged rows: host start, device offset
    uint64_t rows_cap = 0;
    uint32_t *stage = nullptr;  // the ball's rows copied from host memory
    uint64_t stage_cap = 0;
    void *cub_tmp = nullptr;
    size_t cub_cap = 0;

  private:
    int grow_roots(uint64_t need);
    int grow_rows(uint64_t need);
};

}  // namespace g2rt
