// worker_main.cpp - g2_worker, the drop-in for the reference's `bk` and `run`
// binaries (app_BK/main.cu, app_gmatch/main.cu -> Worker<App>::run,
// system/worker.h:28-280).
//
// Same flags and result lines:
//   -dg <graph.bin>   data graph (.bin CSR, ids in degeneracy order for BK)
//   -q  <id>          query preset; 1000 (default) = maximal clique enumeration
//   -h  <hop>         view-bin hop for BK (GMatch takes the plan's hop; must be unset)
//   -cn <n>           consumers = GPUs 0..n-1
//   -ss <0|1>         sort the sources of each bin
//   -prep 1 [-o out.bin]  the reference's preprocess tool: the graph (a SNAP .txt
//                     edge list, deduplicated, no self loops or isolated
//                     vertices) written as <prefix>.bin; any mode reads .txt so
//   -recode 1 -o out.bin [-nb k]   the reference's kcore tool for a .bin input:
//                     degeneracy order + recode to out.bin, k shell bins in
//                     out.bin.2.hop.vbmap; no GPU is used
//   -plan <0|1>       only plan view bins (-m GB each, -ds/-dr applied) and write
//                     them to the .vbmap the other modes read; no GPU is used
//   -ooc <0|1>        out of core: the CSR stays in host memory and each bin's view
//                     is built by -pn host threads and uploaded (g2_view_mce /
//                     g2_view_match); without a .vbmap, bins of at most -m GB
//                     (default 10, the reference's view-bin budget) come from
//                     g2_view_bins
//   -t <threads>      host threads for view building and bin planning
//                     (G2_HOST_THREADS); default: all
//   -qs <k>           -ooc: pinned buffers holding built views (the reference's
//                     view-bin holders; default producers + 2, at least 2)
//   -m, -pn, -dr, -ds, -dst  see below
// Bins come from "<graph.bin>.<hop>.hop.vbmap" (view/view_bin_manager.h:34-94); a
// missing file means one bin holding every vertex.  BK prints one
// "Total No. of Cliques: N" line per bin (app_BK/BK.h:72-76), GMatch one final
// "Total counts: N" (system/worker.h:273-279).
//
// What changes: by default each GPU holds the whole CSR (loaded once) instead of a
// k-hop view per bin, so there is no producer-side materialisation (-pn, -t, -qs, -m
// have no work to size); the view of a bin is a subset of the full graph that
// contains every adjacency list the bin's roots read, so the counts are the same.
// With -ooc 1 the views are materialised as in the reference (a compact induced
// ball per bin, system/worker.h:165-279), for graphs larger than device memory.  Bins go to GPUs
// through an atomic counter instead of the MPMC queues.  -dr (bins by degree sum
// of their roots, largest first) and -ds/-dst (heavy bins cut in two until each
// consumer has -dst more) are applied as the reference applies them
// (g2_view_bins_rebalance); they change the bins, not the totals.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "g2_aimd.h"

namespace {

const char *opt(int argc, char **argv, const char *name, const char *def) {
    for (int i = 1; i + 1 < argc; i++)
        if (!strcmp(argv[i], name)) return argv[i + 1];
    return def;
}

int die(const char *what, int rc) {
    fprintf(stderr, "g2_worker: %s: %s (%d)\n", what, g2_strerror(rc), rc);
    return 1;
}

}  // namespace

int main(int argc, char **argv) {
    const std::string data = opt(argc, argv, "-dg", "");
    const int query = atoi(opt(argc, argv, "-q", "1000"));
    int hop = atoi(opt(argc, argv, "-h", "-1"));
    const int consumers = std::max(1, atoi(opt(argc, argv, "-cn", "1")));
    const int sort_sources = atoi(opt(argc, argv, "-ss", "0"));
    const int reorder = atoi(opt(argc, argv, "-dr", "0"));
    const int do_split = atoi(opt(argc, argv, "-ds", "0"));
    const int split_times = atoi(opt(argc, argv, "-dst", "1"));
    const int ooc = atoi(opt(argc, argv, "-ooc", "0"));
    const int producers = std::max(1, atoi(opt(argc, argv, "-pn", "1")));
    const double mem_gb = atof(opt(argc, argv, "-m", "10"));
    const int plan_only = atoi(opt(argc, argv, "-plan", "0"));
    const int queue_size = std::max(0, atoi(opt(argc, argv, "-qs", "0")));
    const int recode = atoi(opt(argc, argv, "-recode", "0"));
    const int prep = atoi(opt(argc, argv, "-prep", "0"));
    // -t: threads that build views (the reference's ViewBin thread_num) and plan bins
    if (const char *t = opt(argc, argv, "-t", nullptr)) setenv("G2_HOST_THREADS", t, 1);
    const std::string out_bin = opt(argc, argv, "-o", "");
    const uint32_t shell_bins = (uint32_t)std::max(1, atoi(opt(argc, argv, "-nb", "1")));
    if (data.empty()) {
        fprintf(stderr, "usage: g2_worker -dg graph.bin [-q id] [-h hop] [-cn gpus] [-ss 0|1] [-ooc 0|1 -pn threads -m GB] [-plan 1]\n");
        return 2;
    }
    // a .txt graph is a SNAP edge list, read and preprocessed as the reference's
    // preprocess tool does (kmeans/preprocess.cpp); every other name is a .bin
    const bool snap = data.size() > 4 && data.compare(data.size() - 4, 4, ".txt") == 0;
    auto read_graph = [&](uint64_t **rp, uint32_t **ci, uint64_t *n, uint64_t *m) {
        return snap ? g2_read_snap(data.c_str(), 1, rp, ci, n, m) : g2_read_bin(data.c_str(), rp, ci, n, m);
    };
    if (prep) {
        // kmeans/preprocess.cpp: the preprocessed graph as <prefix>.bin (or -o)
        uint64_t *rp = nullptr, n = 0, m = 0;
        uint32_t *ci = nullptr;
        int rc = read_graph(&rp, &ci, &n, &m);
        if (rc) return die(data.c_str(), rc);
        const std::string out = out_bin.empty() ? data.substr(0, data.rfind('.')) + ".bin" : out_bin;
        rc = g2_write_bin(out.c_str(), rp, ci, n, m);
        if (rc) return die(out.c_str(), rc);
        printf("vertex_count=%llu, edge_count=%llu\nwrote %s\n", (unsigned long long)n, (unsigned long long)m,
               out.c_str());
        g2_free(rp);
        g2_free(ci);
        return 0;
    }
    if (recode) {
        // the reference's kcore tool (kmeans/kcore.cpp:230-248) for a .bin input:
        // degeneracy order + recode, the recoded .bin, and -nb shell bins in
        // <out>.2.hop.vbmap; host only
        if (out_bin.empty()) {
            fprintf(stderr, "g2_worker: -recode 1 needs -o <out.bin>\n");
            return 2;
        }
        uint64_t *rp = nullptr, n = 0, m = 0;
        uint32_t *ci = nullptr;
        int rc = read_graph(&rp, &ci, &n, &m);
        if (rc) return die(data.c_str(), rc);
        std::vector<uint32_t> perm(n), core(n), core_new(n), bins(n);
        std::vector<uint64_t> rp2(n + 1);
        std::vector<uint32_t> ci2(m);
        rc = g2_degeneracy_order(rp, ci, n, perm.data(), core.data());
        if (!rc) rc = g2_recode(rp, ci, n, perm.data(), rp2.data(), ci2.data());
        if (rc) return die("degeneracy recode", rc);
        for (uint64_t v = 0; v < n; v++) core_new[perm[v]] = core[v];
        rc = g2_write_bin(out_bin.c_str(), rp2.data(), ci2.data(), n, m);
        if (rc) return die(out_bin.c_str(), rc);
        const std::string vbo = out_bin + ".2.hop.vbmap";
        rc = g2_shell_bins(core_new.data(), n, shell_bins, bins.data());
        if (!rc) rc = g2_write_vbmap(vbo.c_str(), shell_bins, bins.data(), n);
        if (rc) return die(vbo.c_str(), rc);
        printf("vertex_count=%llu, edge_count=%llu, degeneracy=%u\nwrote %s and %s\n", (unsigned long long)n,
               (unsigned long long)m, n ? *std::max_element(core.begin(), core.end()) : 0u, out_bin.c_str(),
               vbo.c_str());
        g2_free(rp);
        g2_free(ci);
        return 0;
    }
    const bool bk = query == 1000;
    g2_plan plan;
    memset(&plan, 0, sizeof(plan));
    if (!bk) {
        if (hop != -1) {
            fprintf(stderr, "g2_worker: -h must be unset for subgraph queries (system/worker.h:61)\n");
            return 2;
        }
        int rc = g2_plan_preset(query, &plan);
        if (rc) return die("query plan", rc);
        hop = (int)plan.hop;
        printf("Hop = %d\nRoot degree = %u\nMatch Order: ", hop, plan.root_degree);
        for (uint32_t i = 0; i < plan.k; i++) printf("%u ", plan.order[i]);
        printf("\n");
    }
    uint64_t *rp = nullptr, n = 0, m = 0;
    uint32_t *ci = nullptr;
    auto t0 = std::chrono::steady_clock::now();
    int rc = read_graph(&rp, &ci, &n, &m);
    if (rc) return die(data.c_str(), rc);
    printf("vertex_count=%llu, edge_count=%llu\n", (unsigned long long)n, (unsigned long long)m);
    // view bins
    std::vector<uint32_t> bins(n, 0);
    uint32_t nbins = 1;
    const std::string vb = data + "." + std::to_string(hop) + ".hop.vbmap";
    // bins of at most -m GB for the query's view shape (MCE: radius 1, full rows)
    auto plan_bins = [&]() {
        uint32_t radius = 1, row_radius = 1, root_degree = 1, flags = 0;
        if (!bk) {
            int r = g2_plan_view_radius(&plan, &radius, &row_radius, &root_degree, &flags);
            if (r) return r;
        }
        int r = g2_view_bins(rp, ci, n, radius, row_radius, root_degree, flags, (uint64_t)(mem_gb * 1e9),
                             bins.data(), &nbins);
        if (!r) printf("view bins: %u (budget %.3f GB)\n", nbins, mem_gb);
        return r;
    };
    if (plan_only || g2_read_vbmap(vb.c_str(), n, &nbins, bins.data()) != G2_OK) {
        nbins = 1;
        std::fill(bins.begin(), bins.end(), 0u);
        if (ooc || plan_only) {
            rc = plan_bins();
            if (rc) return die("view bins", rc);
        }
    }
    // -ds / -dst / -dr: the reference's split of heavy bins over the consumers
    // and heaviest-first order (view/view_bin_manager.h:95-184)
    if (do_split || reorder) {
        rc = g2_view_bins_rebalance(rp, n, bins.data(), nbins, (uint32_t)consumers,
                                    do_split ? (uint32_t)std::max(1, split_times) : 0u, reorder, &nbins);
        if (rc) return die("bin split", rc);
    }
    if (plan_only) {
        // the offline step of the reference's view_pack (kmeans/view_pack.cpp:
        // 290-326): the bins go to the .vbmap that later runs read; no GPU is used
        rc = g2_write_vbmap(vb.c_str(), nbins, bins.data(), n);
        if (rc) return die(vb.c_str(), rc);
        printf("wrote %s\n", vb.c_str());
        g2_free(rp);
        g2_free(ci);
        return 0;
    }
    if (ooc) {
        // consumer c runs bins c, c + cn, ...: its bin_of maps them to 0, 1, ...
        std::atomic<int> failed{0};
        std::atomic<unsigned long long> total{0};
        std::mutex out_mu;
        std::vector<std::thread> th;
        for (int c = 0; c < consumers; c++) {
            th.emplace_back([&, c] {
                std::vector<uint32_t> mine(n, G2_VIEW_NO_BIN);
                uint32_t nb = 0;
                for (uint32_t b = (uint32_t)c; b < nbins; b += (uint32_t)consumers) nb++;
                for (uint64_t v = 0; v < n; v++)
                    if (bins[v] % (uint32_t)consumers == (uint32_t)c) mine[v] = bins[v] / (uint32_t)consumers;
                std::vector<uint64_t> per(std::max<uint32_t>(nb, 1), 0);
                g2_ctx *ctx = nullptr;
                int r = g2_open(c, 0, &ctx);
                if (!r && !bk) r = g2_set_plan(ctx, &plan);
                g2_opts o;
                memset(&o, 0, sizeof(o));
                o.schedule = G2_SCHED_HEURISTIC;
                g2_view_opts vo;
                memset(&vo, 0, sizeof(vo));
                vo.producers = (uint32_t)producers;
                vo.slots = (uint32_t)queue_size;  // -qs: pinned view holders (0 = producers + 2)
                g2_view_stats st;
                memset(&st, 0, sizeof(st));
                uint64_t count = 0;
                if (!r && nb)
                    r = bk ? g2_view_mce(ctx, rp, ci, n, mine.data(), nb, &vo, &o, &count, nullptr, 0, per.data(), &st)
                           : g2_view_match(ctx, rp, ci, n, mine.data(), nb, &vo, &o, &count, per.data(), &st);
                std::lock_guard<std::mutex> lk(out_mu);
                if (r) {
                    fprintf(stderr, "g2_worker: device %d: %s (%d) %s\n", c, g2_strerror(r), r,
                            ctx ? g2_last_cuda_error(ctx) : "");
                    failed = 1;
                } else {
                    total += count;
                    for (uint32_t i = 0; i < nb; i++) {
                        printf("consumer %d completes bin %u\n", c, c + i * (uint32_t)consumers);
                        if (bk) printf("Total No. of Cliques: %llu\n", (unsigned long long)per[i]);
                    }
                    printf("consumer %d: %llu views, %.1f MB uploaded, %.3f ms\n", c, (unsigned long long)st.bins,
                           st.h2d_bytes / 1e6, st.total_ms);
                }
                if (ctx) g2_close(ctx);
            });
        }
        for (auto &t : th) t.join();
        double total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        printf("finish total time, elapsed_time=%.3fms\n", total_ms);
        if (!bk) printf("Total counts: %llu\n", (unsigned long long)total.load());
        g2_free(rp);
        g2_free(ci);
        return failed ? 1 : 0;
    }
    std::vector<std::vector<uint32_t>> sources(nbins);
    for (uint64_t v = 0; v < n; v++) sources[bins[v]].push_back((uint32_t)v);
    if (sort_sources)
        for (auto &s : sources) std::sort(s.begin(), s.end());
    std::vector<uint32_t> order(nbins);  // bins are already numbered heaviest first under -dr / -ds
    for (uint32_t b = 0; b < nbins; b++) order[b] = b;
    std::atomic<uint32_t> next{0};
    std::atomic<int> failed{0};
    std::atomic<unsigned long long> total{0};
    std::mutex out_mu;
    std::vector<std::thread> th;
    for (int c = 0; c < consumers; c++) {
        th.emplace_back([&, c] {
            g2_ctx *ctx = nullptr;
            int r = g2_open(c, 0, &ctx);
            if (!r) r = g2_load_csr(ctx, rp, ci, n, m);
            if (!r) r = g2_reserve(ctx, 0);  // device buffers before the timed runs
            if (!r && !bk) r = g2_set_plan(ctx, &plan);
            for (uint32_t k; !r && (k = next++) < nbins;) {
                const uint32_t b = order[k];
                g2_opts o;
                memset(&o, 0, sizeof(o));
                o.schedule = G2_SCHED_HEURISTIC;
                uint64_t count = 0;
                auto s = std::chrono::steady_clock::now();
                if (sources[b].empty()) {
                    count = 0;
                } else if (bk) {
                    r = g2_mce_run(ctx, sources[b].data(), sources[b].size(), &o, &count, nullptr, 0);
                } else {
                    r = g2_match_run(ctx, sources[b].data(), sources[b].size(), &o, &count);
                }
                double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - s).count();
                if (r) break;
                total += count;
                std::lock_guard<std::mutex> lk(out_mu);
                printf("consumer %d completes bin %u\nfinish In-memory Execution Time, elapsed_time=%.3fms\n", c, b,
                       ms);
                if (bk) printf("Total No. of Cliques: %llu\n", (unsigned long long)count);
                else printf("Currently Total counts: %llu\n", (unsigned long long)total.load());
            }
            if (r) {
                std::lock_guard<std::mutex> lk(out_mu);
                fprintf(stderr, "g2_worker: device %d: %s (%d) %s\n", c, g2_strerror(r), r,
                        ctx ? g2_last_cuda_error(ctx) : "");
                failed = 1;
            }
            if (ctx) g2_close(ctx);
        });
    }
    for (auto &t : th) t.join();
    double total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    printf("finish total time, elapsed_time=%.3fms\n", total_ms);
    if (!bk) printf("Total counts: %llu\n", (unsigned long long)total.load());
    g2_free(rp);
    g2_free(ci);
    return failed ? 1 : 0;
}
