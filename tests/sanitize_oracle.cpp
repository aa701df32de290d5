// sanitize_oracle.cpp - drives the CPU oracle (oracle/g2_oracle.c) through all
// of its entry points so that an AddressSanitizer + UBSan build can check the
// checker itself (tests/test_host_sanitizers.py compiles and runs it).
#include <cstdio>
#include <vector>

#include "g2_aimd.h"

extern "C" {
int orc_mce(const uint64_t *rp, const uint32_t *ci, uint64_t n, const uint32_t *roots, uint64_t nroots, int threads,
            uint64_t *count, uint64_t *hist, uint32_t hist_len, uint64_t *work, uint64_t *root_nodes,
            uint64_t *root_work);
int orc_match(const uint64_t *rp, const uint32_t *ci, uint64_t n, const uint32_t *roots, uint64_t nroots,
              int threads, uint32_t k, const uint32_t *order, const uint32_t *id2order, const uint32_t *bn_count,
              const uint32_t *bn, const uint32_t *cond_count, const uint32_t *cond, uint64_t *count,
              uint64_t *work, uint64_t *root_counts);
int orc_embeddings(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint32_t k, const uint32_t *qadj,
                   uint64_t *out);
int orc_mce_bruteforce(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint64_t *count, uint64_t *hist,
                       uint32_t hist_len);
int64_t orc_kcore(const uint64_t *rp, const uint32_t *ci, uint64_t n, uint32_t *order, uint32_t *core);
}

int main() {
    uint64_t *rp = nullptr, n = 0, m = 0;
    uint32_t *ci = nullptr;
    if (g2_gen_er(600, 0.03, 3, 9, 5, &rp, &ci, &n, &m)) return 1;
    std::vector<uint32_t> perm(n), core(n);
    std::vector<uint64_t> rp2(n + 1);
    std::vector<uint32_t> ci2(m);
    g2_degeneracy_order(rp, ci, n, perm.data(), core.data());
    g2_recode(rp, ci, n, perm.data(), rp2.data(), ci2.data());
    uint64_t count = 0, work = 0;
    std::vector<uint64_t> hist(64), rn(n), rw(n), rc(n);
    if (orc_mce(rp2.data(), ci2.data(), n, nullptr, n, 4, &count, hist.data(), 64, &work, rn.data(), rw.data()))
        return 2;
    printf("mce %llu\n", (unsigned long long)count);
    for (int q : {0, 1, 2, 24}) {
        g2_plan p;
        if (g2_plan_preset(q, &p)) return 3;
        const uint32_t k = p.k;
        std::vector<uint32_t> bn(k * k), cond(k * k * 2), cc(k);
        for (uint32_t i = 0; i < k; i++) {
            for (uint32_t j = 0; j < p.bn_count[i]; j++) bn[i * k + j] = p.bn[i][j];
            cc[i] = p.cond_count[i];
            for (uint32_t j = 0; j < p.cond_count[i]; j++) {
                cond[(i * k + j) * 2] = p.cond[i][j][0];
                cond[(i * k + j) * 2 + 1] = p.cond[i][j][1];
            }
        }
        uint64_t c = 0, w = 0;
        if (orc_match(rp2.data(), ci2.data(), n, nullptr, n, 4, k, p.order, p.id2order, p.bn_count, bn.data(),
                      cc.data(), cond.data(), &c, &w, rc.data()))
            return 4;
        printf("match q%d %llu\n", q, (unsigned long long)c);
    }
    const uint32_t tri[9] = {0, 1, 1, 1, 0, 1, 1, 1, 0};
    uint64_t emb = 0;
    if (orc_embeddings(rp2.data(), ci2.data(), 60, 3, tri, &emb)) return 5;
    uint64_t *rp3 = nullptr, n3 = 0, m3 = 0;
    uint32_t *ci3 = nullptr;
    if (g2_gen_er(40, 0.3, 1, 6, 2, &rp3, &ci3, &n3, &m3)) return 6;
    std::vector<uint64_t> h2(64);
    uint64_t c2 = 0;
    if (orc_mce_bruteforce(rp3, ci3, n3, &c2, h2.data(), 64)) return 7;
    std::vector<uint32_t> order(n), core2(n);
    if (orc_kcore(rp2.data(), ci2.data(), n, order.data(), core2.data()) < 0) return 8;
    g2_free(rp);
    g2_free(ci);
    g2_free(rp3);
    g2_free(ci3);
    printf("oracle ok\n");
    return 0;
}
