"""Query-planner oracle (TEST INFRASTRUCTURE ONLY).

A pure-Python restatement of the reference's query planner, used to check the
library's C++ planner (g2_plan_preset / g2_plan_build).  Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline leg may import it.

Steps restated, with the reference lines they follow:
  query CSR          Graph(QUERY) ctor, common/graph.h:127-156
  ReMapVertexId      common/graph.h:171-266 (BFS from the first max-degree
                     vertex; inside a BFS level sort by degree desc,
                     connections desc, id asc)
  automorphisms      full group of the query (the reference asks bliss for
                     generators and closes them under composition,
                     common/graph.h:575-642; here the group is enumerated
                     directly over all k! permutations, k <= 8)
  GetConditions      common/graph.h:644-686
  SetConditions      common/graph.h:689-699
  FindRoot           system/plan.h:16-73
  GenerateSearchSequence           system/plan.h:75-123
  GenerateBackwardNeighbor         system/plan.h:125-181
  GeneratePreAfterBackwardNeighbor system/plan.h:183-214
  GenerateUsefulOrder              system/plan.h:216-325 (unsigned arithmetic on
                     positions kept: for the root, position-1 wraps, so its
                     pre-condition list covers every vertex, itself included)
  GenerateStoreStrategy            system/plan.h:327-372

Parity: pinned against the reference planner's own output
(tests/golden/plans.json, produced by oracle/_ref/ref_plan built from the
reference sources; see tests/golden/make_plans.py).
"""
from __future__ import annotations

import itertools
from collections import deque

LESS_THAN, LARGER_THAN, NON_EQUAL = 0, 1, 2
EXPAND, PREFIX, COUNT = 0, 1, 2
U32 = 0xFFFFFFFF

# Preset query patterns as undirected edge lists over 0..k-1; the same shapes as
# selectPresetPatterns (common/graph.h:813-1104).
PRESETS = {
    0: (3, [(0, 1), (0, 2), (1, 2)]),                                   # triangle
    1: (4, [(0, 1), (0, 3), (1, 2), (2, 3)]),                           # square
    2: (4, [(0, 1), (0, 2), (0, 3), (1, 2), (2, 3)]),                   # chordal square
    3: (5, [(0, 1), (0, 2), (1, 2), (2, 3), (3, 4)]),                   # 2 tails triangle
    4: (5, [(0, 1), (0, 2), (1, 2), (1, 3), (2, 4), (3, 4)]),           # house
    5: (5, [(0, 1), (0, 2), (0, 3), (0, 4), (1, 2), (1, 3), (2, 3), (3, 4)]),   # chordal house
    6: (5, [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 4), (3, 4)]),   # chordal roof
    7: (5, [(0, 1), (0, 2), (0, 3), (0, 4), (1, 3), (1, 2), (2, 4)]),   # three triangles
    8: (5, [(0, 1), (0, 2), (0, 3), (0, 4), (1, 2), (1, 4), (2, 3), (3, 4)]),   # solar square
    9: (5, [(0, 1), (0, 2), (0, 3), (0, 4), (1, 2), (1, 3), (1, 4), (2, 3), (3, 4)]),  # near 5 clique
    10: (6, [(0, 1), (0, 2), (0, 3), (0, 4), (0, 5), (1, 2), (2, 3), (3, 4), (4, 5)]),  # four triangles
    11: (6, [(0, 1), (0, 2), (0, 3), (0, 5), (1, 2), (1, 3), (1, 4), (2, 4), (2, 5)]),  # one in three triangles
    12: (6, [(0, 1), (0, 2), (1, 2), (1, 3), (1, 4), (1, 5), (2, 3), (2, 4), (2, 5), (3, 4), (4, 5)]),  # near 6 clique
    13: (6, [(0, 1), (0, 2), (1, 3), (2, 3), (2, 4), (2, 5), (3, 4), (3, 5)]),  # square on top
    14: (7, [(0, 1), (0, 2), (0, 3), (0, 4), (0, 5), (1, 2), (1, 3), (1, 5), (2, 3), (2, 5),
             (3, 4), (3, 5), (3, 6), (4, 5), (5, 6)]),                   # near 7 clique
    15: (7, [(0, 1), (0, 2), (0, 3), (0, 4), (1, 2), (1, 3), (1, 4), (2, 3), (2, 4), (3, 4),
             (3, 5), (3, 6), (4, 5), (4, 6)]),                           # 5 clique on top
    16: (5, [(0, 1), (0, 2), (1, 3), (2, 4), (3, 4)]),                   # 5 cycle
    17: (6, [(0, 1), (0, 2), (1, 3), (2, 4), (3, 5), (4, 5)]),           # 6 cycle
    18: (6, [(0, 1), (0, 2), (0, 4), (1, 2), (1, 5), (2, 3), (3, 4), (3, 5), (4, 5)]),  # hourglass
    23: (3, [(0, 1), (0, 2), (1, 2)]),                                   # 3 clique
    24: (4, [(a, b) for a in range(4) for b in range(a + 1, 4)]),        # 4 clique
    25: (5, [(a, b) for a in range(5) for b in range(a + 1, 5)]),        # 5 clique
    26: (6, [(a, b) for a in range(6) for b in range(a + 1, 6)]),        # 6 clique
    27: (7, [(a, b) for a in range(7) for b in range(a + 1, 7)]),        # 7 clique
}


def _adj_lists(k, edges):
    adj = [set() for _ in range(k)]
    for a, b in edges:
        adj[a].add(b)
        adj[b].add(a)
    return [sorted(s) for s in adj]


def remap(k, adj):
    """ReMapVertexId (common/graph.h:171-266)."""
    deg = [len(a) for a in adj]
    root, best = 0, 0
    for i in range(k):
        if deg[i] > best:
            best, root = deg[i], i
    visited = [False] * k
    visited[root] = True
    q = deque([root])
    old_to_new = [0] * k
    new_id = 0
    while q:
        size = len(q)
        level = []
        for _ in range(size):
            f = q.popleft()
            level.append(f)
            for ne in adj[f]:
                if not visited[ne]:
                    visited[ne] = True
                    q.append(ne)
        weights = []
        for v in level:
            conn = sum(1 for ne in adj[v] if visited[ne])
            weights.append((deg[v], conn, v))
        weights.sort(key=lambda t: (-t[0], -t[1], t[2]))
        for _, _, v in weights:
            old_to_new[v] = new_id
            new_id += 1
    nadj = [[] for _ in range(k)]
    for v in range(k):
        nadj[old_to_new[v]] = sorted(old_to_new[u] for u in adj[v])
    return nadj


def automorphisms(k, adj):
    es = {(a, b) for a in range(k) for b in adj[a]}
    out = []
    for p in itertools.permutations(range(k)):
        if all((p[a], p[b]) in es for (a, b) in es):
            out.append(list(p))
    return out


def _eclasses(k, aut):
    ecl = {}
    for i in range(k):
        e = {perm[i] for perm in aut}
        rep = min(e)
        ecl.setdefault(rep, set()).update(e)
    return dict(sorted(ecl.items()))


def conditions(k, adj):
    """GetConditions (common/graph.h:658-686) on the full automorphism group."""
    aut = automorphisms(k, adj)
    ecl = _eclasses(k, aut)
    result = []

    def first_big(ec):
        for rep, s in ec.items():
            if len(s) > 1:
                return s
        return None

    ec = first_big(ecl)
    while ec is not None:
        srt = sorted(ec)
        n0 = srt[0]
        rest = srt[1:]
        for perm in aut:
            m = min(rest, key=lambda n: perm[n])  # first minimum in ascending order
            result.append((n0, m))
        aut = [perm for perm in aut if perm[n0] == n0]
        ecl = _eclasses(k, aut)
        ec = first_big(ecl)
    return sorted(set(result))


def _min_hop(adj, root):
    k = len(adj)
    visited = [False] * k
    level = [-1] * k
    q = deque([root])
    visited[root] = True
    level[root] = 0
    max_v = max_e = -1
    while q:
        f = q.popleft()
        max_v = level[f]
        for j in adj[f]:
            if not visited[j]:
                visited[j] = True
                level[j] = level[f] + 1
                q.append(j)
            elif level[j] == level[f]:
                max_e = level[j]
    return max_v + (1 if max_v == max_e else 0)


def build_plan(k, edges):
    """Full planner: returns a dict with the same fields as tests/golden/plans.json."""
    adj = remap(k, _adj_lists(k, edges))
    deg = [len(a) for a in adj]
    conds = conditions(k, adj)
    order_ = [[] for _ in range(k)]
    for a, b in conds:
        order_[a].append((LESS_THAN, b))
        order_[b].append((LARGER_THAN, a))
    # FindRoot
    root, hop, root_degree = 0, 10, 0
    for u in range(k):
        t = _min_hop(adj, u)
        if t < hop:
            root, hop, root_degree = u, t, deg[u]
        elif t == hop and root_degree < deg[u]:
            root, hop, root_degree = u, t, deg[u]
    # GenerateSearchSequence
    weights = [None] * k
    visited = [False] * k
    visited[root] = True
    q = deque([root])
    h = 0
    weights[root] = (0, deg[root], root)
    while q:
        h += 1
        for _ in range(len(q)):
            f = q.popleft()
            for j in adj[f]:
                if not visited[j]:
                    visited[j] = True
                    q.append(j)
                    weights[j] = (h, deg[j], j)
    weights.sort(key=lambda t: (t[0], -t[1], t[2]))
    seq = [w[2] for w in weights]
    rev = [0] * k
    for i, w in enumerate(seq):
        rev[w] = i
    # GenerateBackwardNeighbor
    bn = [[] for _ in range(k)]
    parent = [0] * k
    vis = [False] * k
    vis[seq[0]] = True
    for i in range(1, k):
        v = seq[i]
        for nv in adj[v]:
            if vis[nv]:
                bn[i].append(nv)
                parent[i] = nv
        vis[v] = True
    share = [0] * k
    for i in range(1, k):
        if len(bn[i]) > 2:
            share[i] = 1
        elif len(bn[i]) == 2 and bn[i][0] != seq[i - 1] and bn[i][1] != seq[i - 1]:
            share[i] = 1
    # GeneratePreAfterBackwardNeighbor
    pre_bn = [[] for _ in range(k)]
    after_bn = [[] for _ in range(k)]
    for i in range(2, k):
        if share[i]:
            v = seq[i]
            for nv in adj[v]:
                if rev[nv] < rev[v] - 1:
                    pre_bn[i].append(nv)
                elif rev[nv] == rev[v] - 1:
                    after_bn[i].append(nv)

    # GenerateUsefulOrder (position arithmetic is unsigned 32-bit in the reference)
    def cond_list(pred):
        out = [[] for _ in range(k)]
        for i in range(k):
            for j in range(k):
                if pred(i, j):
                    hit = next((op for (op, s) in order_[i] if s == j), None)
                    out[i].append([hit if hit is not None else NON_EQUAL, j])
        return out

    cond = cond_list(lambda i, j: rev[i] > rev[j])
    pre_cond = cond_list(lambda i, j: ((rev[i] - 1) & U32) > rev[j])
    after_cond = cond_list(lambda i, j: ((rev[i] - 1) & U32) == rev[j])
    # GenerateStoreStrategy
    strategy = [PREFIX if share[i] else EXPAND for i in range(k)] + [COUNT]
    moving = [1] * k
    for i in range(1, k):
        cnt = 1
        for j in range(i + 1, k):
            if len(bn[i]) == len(bn[j]) and bn[i] == bn[j]:
                cnt += 1
            else:
                break
        moving[i] = cnt
    return {
        "k": k, "hop": hop, "root_degree": root_degree, "adj": adj,
        "conditions": [list(c) for c in conds], "order": seq, "id2order": rev,
        "bn_count": [len(b) for b in bn], "bn": bn, "share": share,
        "pre_bn": pre_bn, "after_bn": after_bn, "cond": cond, "pre_cond": pre_cond,
        "after_cond": after_cond, "strategy": strategy, "moving_lvl": moving,
    }


def preset_plan(q):
    k, edges = PRESETS[q]
    p = build_plan(k, edges)
    p["query"] = q
    return p


def aut_size(k, edges):
    return len(automorphisms(k, _adj_lists(k, edges)))
