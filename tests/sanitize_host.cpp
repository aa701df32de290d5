// sanitize_host.cpp - drives the host graph and planner code of the library
// (generators, .bin / .vbmap / SNAP I/O, degeneracy order and recode, the
// query planner for every preset and a built query) so that sanitizer builds
// can check it (tests/test_host_sanitizers.py compiles and runs it).
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "g2_aimd.h"

static int fail(const char *what) {
    fprintf(stderr, "%s failed\n", what);
    return 1;
}

int main(int argc, char **argv) {
    const std::string dir = argc > 1 ? argv[1] : ".";
    uint64_t *rp = nullptr, n = 0, m = 0;
    uint32_t *ci = nullptr;
    if (g2_gen_rmat(12, 8, 0.57, 0.19, 0.19, 3, 6, 12, 5, &rp, &ci, &n, &m)) return fail("rmat");
    std::vector<uint32_t> perm(n), core(n), bins(n);
    std::vector<uint64_t> rp2(n + 1);
    std::vector<uint32_t> ci2(m);
    if (g2_degeneracy_order(rp, ci, n, perm.data(), core.data())) return fail("order");
    if (g2_recode(rp, ci, n, perm.data(), rp2.data(), ci2.data())) return fail("recode");
    const std::string bin = dir + "/g.bin", vb = dir + "/g.bin.2.hop.vbmap", txt = dir + "/g.txt";
    if (g2_write_bin(bin.c_str(), rp2.data(), ci2.data(), n, m)) return fail("write bin");
    for (uint64_t v = 0; v < n; v++) bins[v] = (uint32_t)(v % 5);
    if (g2_write_vbmap(vb.c_str(), 5, bins.data(), n)) return fail("write vbmap");
    uint64_t *rp3 = nullptr, n3 = 0, m3 = 0;
    uint32_t *ci3 = nullptr, nb = 0;
    if (g2_read_bin(bin.c_str(), &rp3, &ci3, &n3, &m3) || n3 != n || m3 != m) return fail("read bin");
    if (g2_read_vbmap(vb.c_str(), n, &nb, bins.data()) || nb != 5) return fail("read vbmap");
    FILE *f = fopen(txt.c_str(), "w");
    if (!f) return fail("open txt");
    fprintf(f, "# comment\n");
    for (uint64_t v = 0; v < n; v++)
        for (uint64_t e = rp[v]; e < rp[v + 1]; e++) fprintf(f, "%llu\t%u\n", (unsigned long long)v + 3, ci[e] + 3);
    fprintf(f, "7 7\n");
    fclose(f);
    uint64_t *rp4 = nullptr, n4 = 0, m4 = 0;
    uint32_t *ci4 = nullptr;
    for (int pre = 0; pre < 2; pre++) {
        if (g2_read_snap(txt.c_str(), pre, &rp4, &ci4, &n4, &m4)) return fail("read snap");
        g2_free(rp4);
        g2_free(ci4);
    }
    uint64_t *rp5 = nullptr, n5 = 0, m5 = 0;
    uint32_t *ci5 = nullptr;
    if (g2_gen_er(500, 0.05, 2, 8, 3, &rp5, &ci5, &n5, &m5)) return fail("er");
    g2_free(rp5);
    g2_free(ci5);
    if (g2_gen_chunglu(3000, 2.3, 10.0, 4, &rp5, &ci5, &n5, &m5)) return fail("chunglu");
    g2_free(rp5);
    g2_free(ci5);
    g2_plan plan;
    int presets = 0;
    for (int q = 0; q < 40; q++)
        if (g2_plan_preset(q, &plan) == G2_OK) presets++;
    const uint32_t edges[] = {0, 1, 1, 2, 2, 3, 3, 4, 4, 0, 0, 2};  // a 5-cycle with a chord
    if (g2_plan_build(5, edges, 6, &plan)) return fail("plan build");
    g2_free(rp);
    g2_free(ci);
    g2_free(rp3);
    g2_free(ci3);
    printf("host ok: n %llu m %llu, %d presets\n", (unsigned long long)n, (unsigned long long)m, presets);
    return 0;
}
