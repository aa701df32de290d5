// view_run.cu - out-of-core enumeration over view bins behind g2_view_mce /
// g2_view_match (include/g2_aimd.h).  Replaces the reference's producer /
// consumer loop (system/worker.h:165-279): host threads build the views of the
// bins (csrc/host/view_host.cpp) into pinned slots, the calling thread uploads
// each into one of two device slots on a copy stream and runs the ordinary
// enumeration over it on the legacy stream, the next upload overlapping the
// current run.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <vector>

#include "g2_aimd.h"
#include "host/view_host.h"
#include "runtime_internal.h"
#include "view_device.h"

using namespace g2rt;

namespace {

double ms_between(std::chrono::steady_clock::time_point a, std::chrono::steady_clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// A view that a producer thread built in a pinned host slot (slot < 0: the bin
// kept no root; nothing to run).
struct ReadyView {
    uint32_t bin = 0;
    int slot = -1;
    g2view::Sizes sizes;
};

// Producers build the views of the bins, in bin order as threads free up, into
// pinned host slots; the calling thread takes them in the order they are done
// (replaces the MPMC holder queues of system/worker.h:179-236).
struct ViewProducers {
    const uint64_t *rp = nullptr;
    const uint32_t *ci = nullptr;
    uint64_t n = 0;
    const uint64_t *bin_start = nullptr;  // roots of bin b: roots[bin_start[b] .. bin_start[b+1])
    const uint32_t *roots = nullptr;
    uint32_t nbins = 0;
    unsigned build_threads = 1;  // threads of each producer's builder (large views)
    g2view::Shape shape;
    int device = 0;

    std::vector<std::pair<void *, uint64_t>> *slots = nullptr;  // pinned, owned by the context
    std::mutex mu;
    std::condition_variable cv;
    std::vector<int> free_slots;
    std::deque<ReadyView> ready;
    std::atomic<uint32_t> next_bin{0};
    uint32_t running = 0;
    bool stop = false;
    int error = G2_OK;
    double build_ms = 0;
    std::vector<std::thread> threads;

    void start(uint32_t producers, uint32_t nslots) {
        // buffers kept from earlier calls beyond this call's count are released
        // (nothing is in flight yet), so `nslots` bounds the pinned memory
        for (size_t i = nslots; i < slots->size(); i++)
            if ((*slots)[i].first) cudaFreeHost((*slots)[i].first);
        slots->resize(nslots, {nullptr, 0});
        for (uint32_t i = 0; i < nslots; i++) free_slots.push_back((int)i);
        running = producers;
        for (uint32_t t = 0; t < producers; t++) threads.emplace_back([this] { produce(); });
    }

    void fail(int rc) {
        std::lock_guard<std::mutex> g(mu);
        if (error == G2_OK) error = rc;
        stop = true;
        cv.notify_all();
    }

    void produce() {
        try {
            cudaSetDevice(device);  // pinned allocations are made by this thread
            g2view::Builder b(rp, ci, n, build_threads);
            for (;;) {
                const uint32_t bin = next_bin.fetch_add(1);
                if (bin >= nbins) break;
                {
                    std::lock_guard<std::mutex> g(mu);
                    if (stop) break;
                }
                const auto t0 = std::chrono::steady_clock::now();
                ReadyView v;
                v.bin = bin;
                v.sizes = b.plan(roots + bin_start[bin], bin_start[bin + 1] - bin_start[bin], shape);
                if (v.sizes.nsrc) {
                    const g2view::Layout L(v.sizes);
                    {
                        std::unique_lock<std::mutex> g(mu);
                        cv.wait(g, [&] { return stop || !free_slots.empty(); });
                        if (stop) break;
                        v.slot = free_slots.back();
                        free_slots.pop_back();
                    }
                    void *buf = nullptr;
                    uint64_t want = 0;
                    {
                        std::lock_guard<std::mutex> g(mu);  // slot sizes are read by every producer
                        buf = (*slots)[v.slot].first;
                        if ((*slots)[v.slot].second < L.bytes) {
                            // straight to the largest slot so far: slots settle after one call
                            want = std::max<uint64_t>(L.bytes, (*slots)[v.slot].second * 3 / 2);
                            for (const auto &o : *slots) want = std::max(want, o.second);
                            (*slots)[v.slot] = {nullptr, 0};
                        }
                    }
                    if (want) {
                        if (buf) cudaFreeHost(buf);
                        buf = nullptr;
                        if (cudaHostAlloc(&buf, want, cudaHostAllocPortable) != cudaSuccess) {
                            cudaGetLastError();
                            fail(G2_ERR_OOM);
                            break;
                        }
                        std::lock_guard<std::mutex> g(mu);
                        (*slots)[v.slot] = {buf, want};
                    }
                    b.fill_packed(buf, v.sizes);
                }
                const double ms = ms_between(t0, std::chrono::steady_clock::now());
                std::lock_guard<std::mutex> g(mu);
                build_ms += ms;
                ready.push_back(v);
                cv.notify_all();
            }
        } catch (...) {
            fail(G2_ERR_OOM);
        }
        std::lock_guard<std::mutex> g(mu);
        running--;
        cv.notify_all();
    }

    // Next built view, in completion order; false when every bin is done (or on error).
    bool take(ReadyView *v, double *wait_ms) {
        const auto t0 = std::chrono::steady_clock::now();
        std::unique_lock<std::mutex> g(mu);
        cv.wait(g, [&] { return stop || !ready.empty() || running == 0; });
        *wait_ms += ms_between(t0, std::chrono::steady_clock::now());
        if (stop || ready.empty()) return false;
        *v = ready.front();
        ready.pop_front();
        return true;
    }

    void release(int slot) {
        if (slot < 0) return;
        std::lock_guard<std::mutex> g(mu);
        free_slots.push_back(slot);
        cv.notify_all();
    }

    ~ViewProducers() {
        {
            std::lock_guard<std::mutex> g(mu);
            stop = true;
            cv.notify_all();
        }
        for (auto &t : threads) t.join();
    }
};

// Device side of a view run: two device slots, a copy stream, and the events
// that order uploads against the enumeration on the legacy stream.
struct ViewDevice {
    g2_ctx *ctx;
    void **buf;       // the context's two device slots
    uint64_t *cap;
    cudaStream_t copy = nullptr;
    cudaEvent_t copied[2] = {nullptr, nullptr}, done[2] = {nullptr, nullptr};
    cudaEvent_t t_copy[2][2] = {{nullptr, nullptr}, {nullptr, nullptr}};  // around each slot's upload
    cudaEvent_t t_run[2] = {nullptr, nullptr};                             // around the current run
    explicit ViewDevice(g2_ctx *c) : ctx(c), buf(c->view_dev), cap(c->view_dev_cap) {}

    int init() {
        G2_TRY(cudaStreamCreateWithFlags(&copy, cudaStreamNonBlocking));
        for (int d = 0; d < 2; d++) {
            G2_TRY(cudaEventCreateWithFlags(&copied[d], cudaEventDisableTiming));
            G2_TRY(cudaEventCreateWithFlags(&done[d], cudaEventDisableTiming));
            G2_TRY(cudaEventCreate(&t_copy[d][0]));
            G2_TRY(cudaEventCreate(&t_copy[d][1]));
            G2_TRY(cudaEventCreate(&t_run[d]));
        }
        return G2_OK;
    }

    // Device milliseconds of slot d's last upload and of the last run (both ended).
    float copy_ms(int d) const {
        float ms = 0.f;
        return cudaEventElapsedTime(&ms, t_copy[d][0], t_copy[d][1]) == cudaSuccess ? ms : 0.f;
    }
    float run_ms() const {
        float ms = 0.f;
        return cudaEventElapsedTime(&ms, t_run[0], t_run[1]) == cudaSuccess ? ms : 0.f;
    }

    // Upload a built view into device slot d once that slot's last run is done.
    int upload(const ReadyView &v, const void *host, int d) {
        const g2view::Layout L(v.sizes);
        if (cap[d] < L.bytes) {
            const uint64_t want = std::max<uint64_t>(L.bytes, cap[d] + cap[d] / 2);
            if (buf[d]) cudaFree(buf[d]);  // synchronises: the slot's last run has ended anyway
            buf[d] = nullptr;
            cap[d] = 0;
            G2_TRY(cudaMalloc(&buf[d], want));
            cap[d] = want;
        }
        G2_TRY(cudaStreamWaitEvent(copy, done[d], 0));
        G2_TRY(cudaEventRecord(t_copy[d][0], copy));
        G2_TRY(cudaMemcpyAsync(buf[d], host, L.bytes, cudaMemcpyHostToDevice, copy));
        G2_TRY(cudaEventRecord(t_copy[d][1], copy));
        G2_TRY(cudaEventRecord(copied[d], copy));
        return G2_OK;
    }

    // Point the context's graph at device slot d (after its upload) and return
    // the view's sources there.
    uint32_t *bind(const ReadyView &v, int d) {
        const g2view::Layout L(v.sizes);
        char *b = static_cast<char *>(buf[d]);
        ctx->d_rp = reinterpret_cast<uint64_t *>(b);
        ctx->d_fo = reinterpret_cast<uint32_t *>(b + L.fo);
        ctx->d_ci = reinterpret_cast<uint32_t *>(b + L.ci);
        ctx->owns_csr = false;
        ctx->n = v.sizes.n;
        ctx->m = v.sizes.m;
        ctx->max_fwd = v.sizes.max_fwd;
        ctx->batch_off.clear();
        ctx->feat_valid = false;
        ctx->core_loaded = false;
        return reinterpret_cast<uint32_t *>(b + L.src);
    }

    ~ViewDevice() {
        if (copy) cudaStreamSynchronize(copy);
        cudaDeviceSynchronize();
        for (int d = 0; d < 2; d++) {
            if (copied[d]) cudaEventDestroy(copied[d]);
            if (done[d]) cudaEventDestroy(done[d]);
        }
        for (int d = 0; d < 2; d++) {
            for (auto e : t_copy[d])
                if (e) cudaEventDestroy(e);
            if (t_run[d]) cudaEventDestroy(t_run[d]);
        }
        if (copy) cudaStreamDestroy(copy);
    }
};

// One run over a view bound to the context: enqueue (returns before the
// enumeration ends) and finish (waits, spills, reads the results).
struct ViewJob {
    bool mce;
    uint32_t hist_len;  // MCE histogram entries read per view (0: count only)
    g2_opts o{};
    std::vector<unsigned long long> h;

    int enqueue(g2_ctx *ctx, const uint32_t *d_src, uint64_t nsrc) {
        TaskList tl;
        const uint64_t warps = mce ? mce_warps(ctx, &o) : match_warps(ctx, &o);
        int rc = prepare_tasks(ctx, d_src, nsrc, true, &o, warps, nullptr, &tl, mce);
        if (rc) return rc;
        ctx->last_split = tl.split;
        ctx->last_cap = tl.cap;
        rc = grow(ctx, ctx->d_out, ctx->out_cap, 1 + (mce ? hist_len : 0u), "out");
        if (rc) return rc;
        return mce ? mce_enqueue(ctx, tl, &o, ctx->d_out, hist_len, nullptr, nullptr, nullptr)
                   : match_enqueue(ctx, tl, &o, ctx->d_out, nullptr, nullptr, nullptr);
    }

    int finish(g2_ctx *ctx) {
        if (mce) {
            const int rc = mce_host_spill(ctx, nullptr);
            if (rc) return rc;
        }
        h.assign(1 + (mce ? hist_len : 0u), 0ull);
        int status = 0;
        G2_TRY(cudaMemcpy(h.data(), ctx->d_out, sizeof(unsigned long long) * h.size(), cudaMemcpyDeviceToHost));
        G2_TRY(cudaMemcpy(&status, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost));
        return status_to_code(status);
    }
};

int view_run(g2_ctx *ctx, bool mce, const uint64_t *rp, const uint32_t *ci, uint64_t n, const uint32_t *bin_of,
             uint32_t nbins, const g2_view_opts *vo, const g2_opts *opts, uint64_t *count, uint64_t *hist,
             uint32_t hist_len, uint64_t *bin_counts, g2_view_stats *stats) {
    const auto t_start = std::chrono::steady_clock::now();
    if (!ctx || !rp || !bin_of || !count || (hist && !hist_len) || n >= (1ull << 32) || (!ci && rp[n]))
        return G2_ERR_INVALID;
    if (opts && (opts->root_nodes || opts->root_cost || opts->work_bytes || opts->schedule == G2_SCHED_SCORES))
        return G2_ERR_INVALID;
    if (!mce && !ctx->has_plan) return G2_ERR_NO_PLAN;
    // view shape: the query's (MCE: cliques around the root, rows of its
    // neighbours, full balls: X holds the root's smaller neighbours)
    g2view::Shape shape;
    shape.min_deg = 1;
    if (!mce)
        shape = g2view::plan_shape(ctx->plan.k, ctx->plan.bn_count, ctx->plan.bn_pos, ctx->plan.cond_count,
                                   ctx->plan.cond_op, ctx->plan.cond_pos);
    if (vo && vo->radius) shape.radius = vo->radius;
    if (vo && vo->row_radius) shape.row_radius = vo->row_radius;
    if (vo && (vo->flags & G2_VIEW_NO_UPPER)) shape.upper = shape.forward = false;
    if (vo && (vo->flags & G2_VIEW_EGO)) shape.ego = true;
    if (vo && (vo->flags & ~(uint32_t)(G2_VIEW_NO_UPPER | G2_VIEW_EGO | G2_VIEW_DEVICE))) return G2_ERR_INVALID;
    const bool device_build = vo && (vo->flags & G2_VIEW_DEVICE);
    if (device_build && (shape.radius != 1 || shape.row_radius != 1 || shape.ego)) return G2_ERR_UNSUPPORTED;
    if (shape.row_radius > shape.radius || shape.radius > 15) return G2_ERR_INVALID;
    if (shape.ego && (shape.radius != 1 || shape.row_radius != 1)) return G2_ERR_INVALID;
    // roots grouped by bin, ascending inside a bin
    std::vector<uint64_t> start((uint64_t)nbins + 1, 0);
    for (uint64_t v = 0; v < n; v++) {
        if (bin_of[v] == G2_VIEW_NO_BIN) continue;
        if (bin_of[v] >= nbins) return G2_ERR_INVALID;
        start[bin_of[v] + 1]++;
    }
    uint64_t max_roots = 0;
    for (uint32_t b = 0; b < nbins; b++) {
        max_roots = std::max(max_roots, start[b + 1]);
        start[b + 1] += start[b];
    }
    std::vector<uint32_t> roots(start[nbins]);
    {
        std::vector<uint64_t> pos(start.begin(), start.end() - 1);
        for (uint64_t v = 0; v < n; v++)
            if (bin_of[v] != G2_VIEW_NO_BIN) roots[pos[bin_of[v]]++] = (uint32_t)v;
    }
    G2_TRY(cudaSetDevice(ctx->device));
    // the context's own CSR gives way to the view slots
    if (ctx->owns_csr) {
        cudaFree(ctx->d_rp);
        cudaFree(ctx->d_ci);
        ctx->rp_cap = ctx->ci_cap = 0;
    }
    ctx->d_rp = nullptr;
    ctx->d_ci = nullptr;
    ctx->owns_csr = false;
    ctx->n = ctx->m = 0;
    ctx->launches = 0;
    int rc = g2_reserve(ctx, std::max<uint64_t>(max_roots, 1));
    if (rc) return rc;

    ViewJob job;
    job.mce = mce;
    job.hist_len = hist ? hist_len : 0u;
    if (opts) job.o = *opts;
    std::vector<uint64_t> hsum(job.hist_len, 0ull);
    uint64_t total = 0;
    if (bin_counts) memset(bin_counts, 0, sizeof(uint64_t) * nbins);
    g2_view_stats st{};
    uint32_t *saved_fo = ctx->d_fo;
    if (device_build) {
        // the GPU builds each view into a device slot on the copy stream; the
        // next view's build overlaps the current run on the legacy stream
        ViewDevice dev(ctx);
        if (!ctx->view_builder) ctx->view_builder = new DeviceViewBuilder();
        DeviceViewBuilder &vb = *static_cast<DeviceViewBuilder *>(ctx->view_builder);
        struct Unmap {  // the host CSR's mapping ends with the call (device arrays stay)
            DeviceViewBuilder &b;
            ~Unmap() { b.release_host(); }
        } unmap{vb};
        rc = dev.init();
        if (!rc) rc = vb.init(ctx, rp, ci, n, shape);
        int d = 0;
        uint32_t b = 0;
        ReadyView cur, nxt;
        auto build_next = [&](ReadyView *v, int slot) -> int {
            // next bin with a kept source; its view in device slot `slot`
            for (; b < nbins; b++) {
                const auto t0 = std::chrono::steady_clock::now();
                int r = fail_cuda_if(ctx, cudaStreamWaitEvent(dev.copy, dev.done[slot], 0), "view wait");
                if (!r) r = fail_cuda_if(ctx, cudaEventRecord(dev.t_copy[slot][0], dev.copy), "view record");
                g2view::Sizes sz;
                if (!r)
                    r = vb.build(roots.data() + start[b], start[b + 1] - start[b], &dev.buf[slot], &dev.cap[slot],
                                 dev.copy, &sz);
                if (!r) r = fail_cuda_if(ctx, cudaEventRecord(dev.t_copy[slot][1], dev.copy), "view record");
                if (!r) r = fail_cuda_if(ctx, cudaEventRecord(dev.copied[slot], dev.copy), "view record");
                st.build_ms += ms_between(t0, std::chrono::steady_clock::now());
                if (r) return r;
                if (sz.nsrc) {
                    v->bin = b++;
                    v->slot = slot;
                    v->sizes = sz;
                    return G2_OK;
                }
            }
            v->slot = -1;
            return G2_OK;
        };
        if (!rc) rc = build_next(&cur, d);
        while (!rc && cur.slot >= 0) {
            rc = fail_cuda_if(ctx, cudaStreamWaitEvent(nullptr, dev.copied[d], 0), "view wait");
            if (rc) break;
            const uint32_t *d_src = dev.bind(cur, d);
            rc = fail_cuda_if(ctx, cudaEventRecord(dev.t_run[0], nullptr), "view record");
            if (!rc) rc = job.enqueue(ctx, d_src, cur.sizes.nsrc);
            if (!rc) rc = fail_cuda_if(ctx, cudaEventRecord(dev.t_run[1], nullptr), "view record");
            if (!rc) rc = fail_cuda_if(ctx, cudaEventRecord(dev.done[d], nullptr), "view record");
            if (!rc) rc = build_next(&nxt, d ^ 1);
            if (!rc) rc = job.finish(ctx);
            if (rc) break;
            total += job.h[0];
            for (uint32_t s = 0; s < job.hist_len; s++) hsum[s] += job.h[1 + s];
            if (bin_counts) bin_counts[cur.bin] = job.h[0];
            st.bins++;
            st.view_vertices += cur.sizes.n;
            st.view_edges += cur.sizes.m;
            st.max_view_bytes = std::max(st.max_view_bytes, g2view::Layout(cur.sizes).bytes);
            st.copy_ms += dev.copy_ms(d);  // device time of the view's build
            st.run_ms += dev.run_ms();
            cur = nxt;
            d ^= 1;
        }
    } else {
        ViewProducers prod;  // destroyed after dev, whose destructor waits for uploads from its slots
        ViewDevice dev(ctx);
        rc = dev.init();
        prod.rp = rp;
        prod.ci = ci;
        prod.n = n;
        prod.bin_start = start.data();
        prod.roots = roots.data();
        prod.slots = &ctx->view_host;
        prod.nbins = nbins;
        prod.shape = shape;
        prod.device = ctx->device;
        const unsigned cores = g2view::host_threads();
        uint32_t np = vo && vo->producers ? vo->producers : std::min(8u, cores);
        // by default at most 32 GB of builder marks (4 bytes and a bit per vertex each)
        if (!(vo && vo->producers) && n)
            np = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(np, (32ull << 30) / (4 * n + n / 8 + 1)));
        np = std::min<uint32_t>(np, std::max<uint32_t>(nbins, 1u));
        // the host's threads are shared out: few bins get several threads each
        prod.build_threads = std::max(1u, cores / np);
        // the consumer holds one view while it waits for the next: at least 2 slots
        const uint32_t nslots = vo && vo->slots ? std::max<uint32_t>(vo->slots, 2u) : np + 2;
        if (!rc && nbins) prod.start(np, nslots);
        double wait_ms = 0;
        // next view with roots (bins that kept none count 0)
        auto take = [&](ReadyView *v) {
            while (prod.take(v, &wait_ms)) {
                if (v->slot >= 0) return true;
            }
            return false;
        };
        ReadyView cur, nxt;
        int d = 0;
        bool have = !rc && nbins && take(&cur);
        if (have) rc = dev.upload(cur, (*prod.slots)[cur.slot].first, d);
        while (have && !rc) {
            // the run of this view, on the legacy stream after its upload
            rc = fail_cuda_if(ctx, cudaStreamWaitEvent(nullptr, dev.copied[d], 0), "view wait");
            if (rc) break;
            const uint32_t *d_src = dev.bind(cur, d);
            rc = fail_cuda_if(ctx, cudaEventRecord(dev.t_run[0], nullptr), "view record");
            if (!rc) rc = job.enqueue(ctx, d_src, cur.sizes.nsrc);
            if (!rc) rc = fail_cuda_if(ctx, cudaEventRecord(dev.t_run[1], nullptr), "view record");
            if (!rc) rc = fail_cuda_if(ctx, cudaEventRecord(dev.done[d], nullptr), "view record");
            if (rc) break;
            // the next view's upload overlaps this run
            const bool more = take(&nxt);
            if (more) rc = dev.upload(nxt, (*prod.slots)[nxt.slot].first, d ^ 1);
            if (!rc) rc = job.finish(ctx);
            if (rc) break;
            total += job.h[0];
            for (uint32_t s = 0; s < job.hist_len; s++) hsum[s] += job.h[1 + s];
            if (bin_counts) bin_counts[cur.bin] = job.h[0];
            const g2view::Layout L(cur.sizes);
            st.bins++;
            st.view_vertices += cur.sizes.n;
            st.view_edges += cur.sizes.m;
            st.h2d_bytes += L.bytes;
            st.max_view_bytes = std::max(st.max_view_bytes, L.bytes);
            st.copy_ms += dev.copy_ms(d);
            st.run_ms += dev.run_ms();
            prod.release(cur.slot);
            cur = nxt;
            have = more;
            d ^= 1;
        }
        if (!rc) {
            std::lock_guard<std::mutex> g(prod.mu);
            rc = prod.error;
        }
        if (rc) prod.fail(rc);
        for (auto &t : prod.threads) t.join();
        prod.threads.clear();
        st.build_ms = prod.build_ms;
        st.wait_ms = wait_ms;
    }
    ctx->d_fo = saved_fo;
    ctx->d_rp = nullptr;
    ctx->d_ci = nullptr;
    ctx->n = ctx->m = 0;
    if (rc) return rc;
    *count = total;
    if (hist)
        for (uint32_t s = 0; s < hist_len; s++) hist[s] = hsum[s];
    st.total_ms = ms_between(t_start, std::chrono::steady_clock::now());
    if (stats) *stats = st;
    return G2_OK;
}

}  // namespace

extern "C" {

int g2_view_mce(g2_ctx *ctx, const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n, const uint32_t *bin_of,
                uint32_t nbins, const g2_view_opts *vopts, const g2_opts *opts, uint64_t *count, uint64_t *hist,
                uint32_t hist_len, uint64_t *bin_counts, g2_view_stats *stats) {
    return view_run(ctx, true, row_ptrs, cols, n, bin_of, nbins, vopts, opts, count, hist, hist_len, bin_counts,
                    stats);
}

int g2_view_match(g2_ctx *ctx, const uint64_t *row_ptrs, const uint32_t *cols, uint64_t n, const uint32_t *bin_of,
                  uint32_t nbins, const g2_view_opts *vopts, const g2_opts *opts, uint64_t *count,
                  uint64_t *bin_counts, g2_view_stats *stats) {
    return view_run(ctx, false, row_ptrs, cols, n, bin_of, nbins, vopts, opts, count, nullptr, 0, bin_counts, stats);
}


}  // extern "C"
