// ref_plan_dump.cpp - runs the REFERENCE query planner and prints its plan.
//
// Test infrastructure: compiled by oracle/Makefile against the reference's own
// headers (common/graph.h, system/plan.h) and bliss sources, so that the plans
// of this library and of the oracle can be pinned to the reference's output.
// The call sequence is the one in Worker::run (system/worker.h:59-89):
//   Graph("", q, QUERY); SetConditions(GetConditions(GetBlissGraph()));
//   Plan: FindRoot, GenerateSearchSequence, GenerateBackwardNeighbor,
//         GeneratePreAfterBackwardNeighbor, GenerateUsefulOrder,
//         GenerateStoreStrategy.
// Output: one JSON object per query id given on the command line.
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "common/graph.h"
#include "system/plan.h"

static void arr(const char *name, const uintV *a, size_t n, bool last = false) {
    printf("\"%s\": [", name);
    for (size_t i = 0; i < n; i++) printf("%s%u", i ? ", " : "", a[i]);
    printf("]%s", last ? "" : ", ");
}

int main(int argc, char **argv) {
    printf("[");
    for (int a = 1; a < argc; a++) {
        int q = atoi(argv[a]);
        Graph query_G("", (PresetPatternType)q, GraphType::QUERY);
        auto conds = query_G.GetConditions(query_G.GetBlissGraph());
        query_G.SetConditions(conds);
        Plan plan;
        plan.graph = std::move(query_G);
        plan.FindRoot();
        plan.GenerateSearchSequence();
        plan.GenerateBackwardNeighbor();
        plan.GeneratePreAfterBackwardNeighbor();
        plan.GenerateUsefulOrder();
        plan.GenerateStoreStrategy();
        size_t k = plan.vertex_count_;
        printf("%s{\"query\": %d, \"k\": %zu, \"hop\": %d, \"root_degree\": %zu, ", a > 1 ? ", " : "", q, k,
               plan.GetHop(), plan.root_degree_);
        // remapped query graph (after ReMapVertexId)
        printf("\"adj\": [");
        for (size_t u = 0; u < k; u++) {
            printf("%s[", u ? ", " : "");
            for (auto e = plan.graph.GetRowPtrs()[u]; e < plan.graph.GetRowPtrs()[u + 1]; e++)
                printf("%s%u", e > plan.graph.GetRowPtrs()[u] ? ", " : "", plan.graph.GetCols()[e]);
            printf("]");
        }
        printf("], \"conditions\": [");
        for (size_t i = 0; i < conds.size(); i++) printf("%s[%u, %u]", i ? ", " : "", conds[i].first, conds[i].second);
        printf("], ");
        arr("order", plan.seq_.data(), k);
        arr("id2order", plan.reverse_seq_.data(), k);
        arr("bn_count", plan.backNeighborCountHost, k);
        printf("\"bn\": [");
        for (size_t p = 0; p < k; p++) {
            printf("%s[", p ? ", " : "");
            for (size_t j = 0; j < plan.backNeighborCountHost[p]; j++)
                printf("%s%u", j ? ", " : "", plan.backNeighborsHost[p * k + j]);
            printf("]");
        }
        printf("], \"share\": [");
        for (size_t p = 0; p < k; p++) printf("%s%d", p ? ", " : "", plan.share_intersection[p] ? 1 : 0);
        printf("], ");
        auto lists = [&](const char *name, const uintV *cnt, const uintV *vals, bool two) {
            printf("\"%s\": [", name);
            for (size_t p = 0; p < k; p++) {
                printf("%s[", p ? ", " : "");
                for (size_t j = 0; j < cnt[p]; j++) {
                    if (two)
                        printf("%s[%u, %u]", j ? ", " : "", vals[p * k * 2 + 2 * j], vals[p * k * 2 + 2 * j + 1]);
                    else
                        printf("%s%u", j ? ", " : "", vals[p * k + j]);
                }
                printf("]");
            }
            printf("], ");
        };
        // pre/after back neighbours are only defined for positions >= 2 with share
        std::vector<uintV> pre_cnt(k, 0), aft_cnt(k, 0);
        for (size_t p = 2; p < k; p++)
            if (plan.share_intersection[p]) {
                pre_cnt[p] = plan.preBackNeighborCountHost[p];
                aft_cnt[p] = plan.afterBackNeighborCountHost[p];
            }
        lists("pre_bn", pre_cnt.data(), plan.preBackNeighborsHost, false);
        lists("after_bn", aft_cnt.data(), plan.afterBackNeighborsHost, false);
        lists("cond", plan.condNumHost, plan.condOrderHost, true);
        lists("pre_cond", plan.preCondNumHost, plan.preCondOrderHost, true);
        lists("after_cond", plan.afterCondNumHost, plan.afterCondOrderHost, true);
        std::vector<uintV> strat(k + 1);
        for (size_t p = 0; p <= k; p++) strat[p] = (uintV)plan.strategy[p];
        arr("strategy", strat.data(), k + 1);
        arr("moving_lvl", plan.moving_lvl, k, true);
        printf("}");
    }
    printf("]\n");
    return 0;
}
