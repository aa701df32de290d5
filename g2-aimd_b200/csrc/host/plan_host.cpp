// plan_host.cpp - query planner of libg2aimd.so.
//
// Produces the plan arrays the reference builds in Worker::run
// (system/worker.h:59-89) with the same results:
//   query CSR + ReMapVertexId      common/graph.h:127-266
//   symmetry-breaking conditions   common/graph.h:644-699 (GetConditions); the
//       automorphism group is enumerated directly over the k! permutations
//       (k <= 8) instead of asking bliss for generators and closing them under
//       composition (common/graph.h:575-642): both give the full group, and
//       GetConditions depends only on the group.
//   FindRoot .. GenerateStoreStrategy   system/plan.h:16-372
#include <algorithm>
#include <cstring>
#include <deque>
#include <set>
#include <tuple>
#include <vector>

#include "g2_aimd.h"

namespace {

struct Preset {
    int id;
    uint32_t k;
    std::vector<std::pair<uint32_t, uint32_t>> edges;
};

std::vector<std::pair<uint32_t, uint32_t>> clique_edges(uint32_t k) {
    std::vector<std::pair<uint32_t, uint32_t>> e;
    for (uint32_t a = 0; a < k; a++)
        for (uint32_t b = a + 1; b < k; b++) e.push_back({a, b});
    return e;
}

// Shapes of selectPresetPatterns (common/graph.h:813-1104) as edge lists.
const std::vector<Preset> &presets() {
    static const std::vector<Preset> P = {
        {0, 3, {{0, 1}, {0, 2}, {1, 2}}},
        {1, 4, {{0, 1}, {0, 3}, {1, 2}, {2, 3}}},
        {2, 4, {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {2, 3}}},
        {3, 5, {{0, 1}, {0, 2}, {1, 2}, {2, 3}, {3, 4}}},
        {4, 5, {{0, 1}, {0, 2}, {1, 2}, {1, 3}, {2, 4}, {3, 4}}},
        {5, 5, {{0, 1}, {0, 2}, {0, 3}, {0, 4}, {1, 2}, {1, 3}, {2, 3}, {3, 4}}},
        {6, 5, {{0, 1}, {0, 2}, {0, 3}, {1, 2}, {1, 3}, {2, 4}, {3, 4}}},
        {7, 5, {{0, 1}, {0, 2}, {0, 3}, {0, 4}, {1, 3}, {1, 2}, {2, 4}}},
        {8, 5, {{0, 1}, {0, 2}, {0, 3}, {0, 4}, {1, 2}, {1, 4}, {2, 3}, {3, 4}}},
        {9, 5, {{0, 1}, {0, 2}, {0, 3}, {0, 4}, {1, 2}, {1, 3}, {1, 4}, {2, 3}, {3, 4}}},
        {10, 6, {{0, 1}, {0, 2}, {0, 3}, {0, 4}, {0, 5}, {1, 2}, {2, 3}, {3, 4}, {4, 5}}},
        {11, 6, {{0, 1}, {0, 2}, {0, 3}, {0, 5}, {1, 2}, {1, 3}, {1, 4}, {2, 4}, {2, 5}}},
        {12, 6, {{0, 1}, {0, 2}, {1, 2}, {1, 3}, {1, 4}, {1, 5}, {2, 3}, {2, 4}, {2, 5}, {3, 4}, {4, 5}}},
        {13, 6, {{0, 1}, {0, 2}, {1, 3}, {2, 3}, {2, 4}, {2, 5}, {3, 4}, {3, 5}}},
        {14, 7, {{0, 1}, {0, 2}, {0, 3}, {0, 4}, {0, 5}, {1, 2}, {1, 3}, {1, 5}, {2, 3}, {2, 5}, {3, 4}, {3, 5},
                 {3, 6}, {4, 5}, {5, 6}}},
        {15, 7, {{0, 1}, {0, 2}, {0, 3}, {0, 4}, {1, 2}, {1, 3}, {1, 4}, {2, 3}, {2, 4}, {3, 4}, {3, 5}, {3, 6},
                 {4, 5}, {4, 6}}},
        {16, 5, {{0, 1}, {0, 2}, {1, 3}, {2, 4}, {3, 4}}},
        {17, 6, {{0, 1}, {0, 2}, {1, 3}, {2, 4}, {3, 5}, {4, 5}}},
        {18, 6, {{0, 1}, {0, 2}, {0, 4}, {1, 2}, {1, 5}, {2, 3}, {3, 4}, {3, 5}, {4, 5}}},
        {23, 3, clique_edges(3)},
        {24, 4, clique_edges(4)},
        {25, 5, clique_edges(5)},
        {26, 6, clique_edges(6)},
        {27, 7, clique_edges(7)},
    };
    return P;
}

using Adj = std::vector<std::vector<uint32_t>>;

Adj remap(const Adj &adj) {
    const uint32_t k = (uint32_t)adj.size();
    uint32_t root = 0;
    size_t best = 0;
    for (uint32_t i = 0; i < k; i++)
        if (adj[i].size() > best) best = adj[i].size(), root = i;
    std::vector<bool> vis(k, false);
    vis[root] = true;
    std::deque<uint32_t> q{root};
    std::vector<uint32_t> o2n(k);
    uint32_t nid = 0;
    while (!q.empty()) {
        size_t sz = q.size();
        std::vector<uint32_t> lvl;
        for (size_t i = 0; i < sz; i++) {
            uint32_t f = q.front();
            q.pop_front();
            lvl.push_back(f);
            for (uint32_t ne : adj[f])
                if (!vis[ne]) vis[ne] = true, q.push_back(ne);
        }
        std::vector<std::tuple<size_t, size_t, uint32_t>> w;
        for (uint32_t v : lvl) {
            size_t conn = 0;
            for (uint32_t ne : adj[v]) conn += vis[ne];
            w.emplace_back(adj[v].size(), conn, v);
        }
        std::sort(w.begin(), w.end(), [](const auto &a, const auto &b) {
            if (std::get<0>(a) != std::get<0>(b)) return std::get<0>(a) > std::get<0>(b);
            if (std::get<1>(a) != std::get<1>(b)) return std::get<1>(a) > std::get<1>(b);
            return std::get<2>(a) < std::get<2>(b);
        });
        for (auto &t : w) o2n[std::get<2>(t)] = nid++;
    }
    Adj out(k);
    for (uint32_t v = 0; v < k; v++) {
        for (uint32_t u : adj[v]) out[o2n[v]].push_back(o2n[u]);
        std::sort(out[o2n[v]].begin(), out[o2n[v]].end());
    }
    return out;
}

std::vector<std::vector<uint32_t>> automorphisms(const Adj &adj) {
    const uint32_t k = (uint32_t)adj.size();
    std::vector<std::vector<bool>> m(k, std::vector<bool>(k, false));
    for (uint32_t a = 0; a < k; a++)
        for (uint32_t b : adj[a]) m[a][b] = true;
    std::vector<uint32_t> p(k);
    for (uint32_t i = 0; i < k; i++) p[i] = i;
    std::vector<std::vector<uint32_t>> out;
    do {
        bool ok = true;
        for (uint32_t a = 0; a < k && ok; a++)
            for (uint32_t b : adj[a])
                if (!m[p[a]][p[b]]) {
                    ok = false;
                    break;
                }
        if (ok) out.push_back(p);
    } while (std::next_permutation(p.begin(), p.end()));
    return out;
}

std::vector<std::pair<uint32_t, uint32_t>> conditions(const Adj &adj) {
    const uint32_t k = (uint32_t)adj.size();
    auto aut = automorphisms(adj);
    auto first_class = [&](const std::vector<std::vector<uint32_t>> &A) -> std::set<uint32_t> {
        // equivalence classes keyed by their minimum, scanned in key order
        std::vector<std::set<uint32_t>> byrep(k);
        for (uint32_t i = 0; i < k; i++) {
            std::set<uint32_t> e;
            for (auto &perm : A) e.insert(perm[i]);
            byrep[*e.begin()].insert(e.begin(), e.end());
        }
        for (uint32_t r = 0; r < k; r++)
            if (byrep[r].size() > 1) return byrep[r];
        return {};
    };
    std::vector<std::pair<uint32_t, uint32_t>> res;
    auto ec = first_class(aut);
    while (!ec.empty()) {
        uint32_t n0 = *ec.begin();
        for (auto &perm : aut) {
            auto it = std::next(ec.begin());
            uint32_t mn = *it;
            for (; it != ec.end(); ++it)
                if (perm[*it] < perm[mn]) mn = *it;
            res.emplace_back(n0, mn);
        }
        aut.erase(std::remove_if(aut.begin(), aut.end(), [n0](const auto &perm) { return perm[n0] != n0; }),
                  aut.end());
        ec = first_class(aut);
    }
    std::sort(res.begin(), res.end());
    res.erase(std::unique(res.begin(), res.end()), res.end());
    return res;
}

int min_hop(const Adj &adj, uint32_t root) {
    const uint32_t k = (uint32_t)adj.size();
    std::vector<bool> vis(k, false);
    std::vector<int> lvl(k, -1);
    std::deque<uint32_t> q{root};
    vis[root] = true;
    lvl[root] = 0;
    int mv = -1, me = -1;
    while (!q.empty()) {
        uint32_t f = q.front();
        q.pop_front();
        mv = lvl[f];
        for (uint32_t j : adj[f]) {
            if (!vis[j]) vis[j] = true, lvl[j] = lvl[f] + 1, q.push_back(j);
            else if (lvl[j] == lvl[f]) me = lvl[j];
        }
    }
    return mv + (mv == me ? 1 : 0);
}

int plan_from_adj(Adj adj, g2_plan *out) {
    const uint32_t k = (uint32_t)adj.size();
    if (k < 2 || k > G2_MAX_QUERY) return G2_ERR_UNSUPPORTED;
    adj = remap(adj);
    // connectivity check: remap visits only the root's component
    {
        std::vector<bool> vis(k, false);
        std::deque<uint32_t> q{0};
        vis[0] = true;
        uint32_t c = 1;
        while (!q.empty()) {
            uint32_t f = q.front();
            q.pop_front();
            for (uint32_t j : adj[f])
                if (!vis[j]) vis[j] = true, c++, q.push_back(j);
        }
        if (c != k) return G2_ERR_INVALID;
    }
    std::vector<uint32_t> deg(k);
    for (uint32_t i = 0; i < k; i++) deg[i] = (uint32_t)adj[i].size();
    auto conds = conditions(adj);
    std::vector<std::vector<std::pair<uint32_t, uint32_t>>> ord(k);  // (op, vertex)
    for (auto &c : conds) {
        ord[c.first].push_back({G2_COND_LESS_THAN, c.second});
        ord[c.second].push_back({G2_COND_LARGER_THAN, c.first});
    }
    g2_plan p;
    memset(&p, 0, sizeof(p));
    p.k = k;
    // FindRoot
    uint32_t root = 0, rdeg = 0;
    int hop = 10;
    for (uint32_t u = 0; u < k; u++) {
        int t = min_hop(adj, u);
        if (t < hop) root = u, hop = t, rdeg = deg[u];
        else if (t == hop && rdeg < deg[u]) root = u, rdeg = deg[u];
    }
    p.hop = (uint32_t)hop;
    p.root_degree = rdeg;
    // GenerateSearchSequence
    std::vector<std::tuple<int, int, uint32_t>> w(k);
    std::vector<bool> vis(k, false);
    vis[root] = true;
    std::deque<uint32_t> q{root};
    int h = 0;
    w[root] = {0, (int)deg[root], root};
    while (!q.empty()) {
        h++;
        size_t sz = q.size();
        for (size_t i = 0; i < sz; i++) {
            uint32_t f = q.front();
            q.pop_front();
            for (uint32_t j : adj[f])
                if (!vis[j]) vis[j] = true, q.push_back(j), w[j] = {h, (int)deg[j], j};
        }
    }
    std::sort(w.begin(), w.end(), [](const auto &a, const auto &b) {
        if (std::get<0>(a) != std::get<0>(b)) return std::get<0>(a) < std::get<0>(b);
        if (std::get<1>(a) != std::get<1>(b)) return std::get<1>(a) > std::get<1>(b);
        return std::get<2>(a) < std::get<2>(b);
    });
    for (uint32_t i = 0; i < k; i++) {
        p.order[i] = std::get<2>(w[i]);
        p.id2order[p.order[i]] = i;
    }
    // GenerateBackwardNeighbor
    std::vector<bool> seen(k, false);
    seen[p.order[0]] = true;
    for (uint32_t i = 1; i < k; i++) {
        uint32_t v = p.order[i];
        for (uint32_t nv : adj[v])
            if (seen[nv]) p.bn[i][p.bn_count[i]++] = nv, p.parent[i] = nv;
        seen[v] = true;
    }
    for (uint32_t i = 1; i < k; i++) {
        if (p.bn_count[i] > 2) p.share[i] = 1;
        else if (p.bn_count[i] == 2 && p.bn[i][0] != p.order[i - 1] && p.bn[i][1] != p.order[i - 1]) p.share[i] = 1;
    }
    // GeneratePreAfterBackwardNeighbor
    for (uint32_t i = 2; i < k; i++) {
        if (!p.share[i]) continue;
        uint32_t v = p.order[i];
        for (uint32_t nv : adj[v]) {
            if (p.id2order[nv] < p.id2order[v] - 1) p.pre_bn[i][p.pre_bn_count[i]++] = nv;
            else if (p.id2order[nv] == p.id2order[v] - 1) p.after_bn[i][p.after_bn_count[i]++] = nv;
        }
    }
    // GenerateUsefulOrder (unsigned position arithmetic, as the reference)
    auto fill = [&](uint32_t (*cnt)[G2_MAX_QUERY], uint32_t (*lst)[G2_MAX_QUERY][G2_MAX_QUERY][2], int which) {
        for (uint32_t i = 0; i < k; i++)
            for (uint32_t j = 0; j < k; j++) {
                uint32_t ri = p.id2order[i], rj = p.id2order[j];
                bool take = which == 0 ? ri > rj : which == 1 ? (uint32_t)(ri - 1u) > rj : (uint32_t)(ri - 1u) == rj;
                if (!take) continue;
                uint32_t op = G2_COND_NON_EQUAL;
                for (auto &o : ord[i])
                    if (o.second == j) {
                        op = o.first;
                        break;
                    }
                (*lst)[i][(*cnt)[i]][0] = op;
                (*lst)[i][(*cnt)[i]][1] = j;
                (*cnt)[i]++;
            }
    };
    fill(&p.cond_count, &p.cond, 0);
    fill(&p.pre_cond_count, &p.pre_cond, 1);
    fill(&p.after_cond_count, &p.after_cond, 2);
    // GenerateStoreStrategy
    for (uint32_t i = 0; i < k; i++) p.strategy[i] = p.share[i] ? G2_STORE_PREFIX : G2_STORE_EXPAND;
    p.strategy[k] = G2_STORE_COUNT;
    for (uint32_t i = 0; i < k; i++) p.moving_lvl[i] = 1;
    for (uint32_t i = 1; i < k; i++) {
        uint32_t c = 1;
        for (uint32_t j = i + 1; j < k; j++) {
            bool same = p.bn_count[i] == p.bn_count[j];
            for (uint32_t t = 0; same && t < p.bn_count[i]; t++) same = p.bn[i][t] == p.bn[j][t];
            if (!same) break;
            c++;
        }
        p.moving_lvl[i] = c;
    }
    *out = p;
    return G2_OK;
}

}  // namespace

extern "C" {

int g2_plan_build(uint32_t k, const uint32_t *edges, uint32_t nedges, g2_plan *out) {
    if (!out || (!edges && nedges) || k < 2 || k > G2_MAX_QUERY) return G2_ERR_INVALID;
    std::vector<std::set<uint32_t>> s(k);
    for (uint32_t e = 0; e < nedges; e++) {
        uint32_t a = edges[2 * e], b = edges[2 * e + 1];
        if (a >= k || b >= k || a == b) return G2_ERR_INVALID;
        s[a].insert(b);
        s[b].insert(a);
    }
    Adj adj(k);
    for (uint32_t i = 0; i < k; i++) adj[i].assign(s[i].begin(), s[i].end());
    return plan_from_adj(adj, out);
}

int g2_plan_preset(int query_id, g2_plan *out) {
    if (!out) return G2_ERR_INVALID;
    for (const auto &pr : presets())
        if (pr.id == query_id) {
            std::vector<uint32_t> flat;
            for (auto &e : pr.edges) flat.push_back(e.first), flat.push_back(e.second);
            return g2_plan_build(pr.k, flat.data(), (uint32_t)pr.edges.size(), out);
        }
    return G2_ERR_INVALID;
}

}  // extern "C"
