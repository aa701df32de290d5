// tsan_views.cpp - drives the threaded paths of the view builder and the bin
// planner (parallel row passes, the atomic radius-1 walk, the ego filter,
// range-parallel plans) so that a ThreadSanitizer build can check them for
// data races (tests/test_host_tsan.py compiles and runs it).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>
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
    return 0;
}
