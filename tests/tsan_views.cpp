// tsan_views.cpp - drives the threaded paths of the view builder and the bin
// planner (parallel row passes, the atomic radius-1 walk, the ego filter,
// range-parallel plans) so that a ThreadSanitizer build can check them for
// data races (tests/test_host_sanitizers.py compiles and runs it).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>
#include "g2_aimd.h"
#include "host/view_host.h"
int main() {
    // a random power-law-ish symmetric graph, n = 70000 (threaded bin plans need 2^16)
    const uint32_t n = 70000;
    std::mt19937_64 rng(7);
    std::vector<std::vector<uint32_t>> adj(n);
    for (uint32_t e = 0; e < 400000; e++) {
        uint32_t a = (uint32_t)(rng() % n), b = (uint32_t)((rng() % 64) * (rng() % 64) % n);
        if (a == b) continue;
        adj[a].push_back(b); adj[b].push_back(a);
    }
    std::vector<uint64_t> rp(n + 1, 0); std::vector<uint32_t> ci;
    for (uint32_t v = 0; v < n; v++) {
        auto &r = adj[v]; std::sort(r.begin(), r.end()); r.erase(std::unique(r.begin(), r.end()), r.end());
        rp[v + 1] = rp[v] + r.size(); ci.insert(ci.end(), r.begin(), r.end());
    }
    std::vector<uint32_t> src(n); for (uint32_t v = 0; v < n; v++) src[v] = v;
    for (int mode = 0; mode < 4; mode++) {
        g2view::Shape sh; sh.radius = 1; sh.row_radius = 1; sh.min_deg = 1;
        sh.upper = mode >= 1; sh.forward = mode >= 2; sh.ego = mode == 3 || mode == 0;
        g2view::Builder b(rp.data(), ci.data(), n, 6);
        auto s = b.plan(src.data(), n, sh);
        g2view::Layout L(s); std::vector<char> buf(L.bytes);
        b.fill_packed(buf.data(), s);
        std::vector<uint32_t> bins(n);
        uint32_t nb = g2view::plan_bins(rp.data(), ci.data(), n, sh, (8 * (n + 1) + 4 * ci.size()) / 30, bins.data(), 6);
        printf("mode %d view n %llu m %llu bins %u\n", mode, (unsigned long long)s.n, (unsigned long long)s.m, nb);
    }
    // the C entry points: views of radius 2 (serial upper walk), bin split and
    // reorder, shell bins
    std::vector<uint32_t> some(src.begin(), src.begin() + 5000);
    for (uint32_t flags : {0u, (uint32_t)G2_VIEW_UPPER}) {
        g2_view v;
        if (g2_view_materialize(rp.data(), ci.data(), n, some.data(), some.size(), 2, 1, 2, flags, &v) != G2_OK)
            return 1;
        printf("radius-2 view n %llu m %llu\n", (unsigned long long)v.n, (unsigned long long)v.m);
        g2_view_free(&v);
    }
    std::vector<uint32_t> bins(n);
    uint32_t nb = 0;
    if (g2_view_bins(rp.data(), ci.data(), n, 1, 1, 1, 0, 200000, bins.data(), &nb) != G2_OK) return 1;
    if (g2_view_bins_rebalance(rp.data(), n, bins.data(), nb, 4, 2, 1, &nb) != G2_OK) return 1;
    std::vector<uint32_t> core(n);
    for (uint32_t v = 0; v < n; v++) core[v] = v / 1000;  // ascending shells
    if (g2_shell_bins(core.data(), n, 3, bins.data()) != G2_OK) return 1;
    printf("rebalanced bins %u\n", nb);
    return 0;
}
