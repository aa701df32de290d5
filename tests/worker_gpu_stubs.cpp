// worker_gpu_stubs.cpp - stand-ins for the device entry points of libg2aimd.so
// so that g2_worker's host-only modes (-prep, -recode, -plan) can be built with
// sanitizers from the host sources alone (tests/test_host_sanitizers.py).  Any
// call reports G2_ERR_CUDA: the host-only modes must not reach them.
#include "g2_aimd.h"

extern "C" {
const char *g2_strerror(int) { return "stub"; }
const char *g2_last_cuda_error(const g2_ctx *) { return ""; }
int g2_open(int, uint64_t, g2_ctx **) { return G2_ERR_CUDA; }
int g2_close(g2_ctx *) { return G2_ERR_CUDA; }
int g2_load_csr(g2_ctx *, const uint64_t *, const uint32_t *, uint64_t, uint64_t) { return G2_ERR_CUDA; }
int g2_reserve(g2_ctx *, uint64_t) { return G2_ERR_CUDA; }
int g2_set_plan(g2_ctx *, const g2_plan *) { return G2_ERR_CUDA; }
int g2_mce_run(g2_ctx *, const uint32_t *, uint64_t, const g2_opts *, uint64_t *, uint64_t *, uint32_t) {
    return G2_ERR_CUDA;
}
int g2_match_run(g2_ctx *, const uint32_t *, uint64_t, const g2_opts *, uint64_t *) { return G2_ERR_CUDA; }
int g2_view_mce(g2_ctx *, const uint64_t *, const uint32_t *, uint64_t, const uint32_t *, uint32_t,
                const g2_view_opts *, const g2_opts *, uint64_t *, uint64_t *, uint32_t, uint64_t *,
                g2_view_stats *) {
    return G2_ERR_CUDA;
}
int g2_view_match(g2_ctx *, const uint64_t *, const uint32_t *, uint64_t, const uint32_t *, uint32_t,
                  const g2_view_opts *, const g2_opts *, uint64_t *, uint64_t *, g2_view_stats *) {
    return G2_ERR_CUDA;
}
}
