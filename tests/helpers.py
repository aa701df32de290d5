"""Small seeded graphs shared by the tests."""
import numpy as np


def random_graph(G, n, p, seed, planted=()):
    """G(n, p) over numpy's PCG64 plus cliques on the given vertex tuples."""
    rng = np.random.default_rng(seed)
    iu = np.triu_indices(n, 1)
    keep = rng.random(iu[0].size) < p
    edges = list(zip(iu[0][keep].tolist(), iu[1][keep].tolist()))
    for cl in planted:
        cl = list(cl)
        edges += [(cl[i], cl[j]) for i in range(len(cl)) for j in range(i + 1, len(cl))]
    return G.from_edges(n, edges, name=f"gnp{n}_{p}_{seed}")


def small_graphs(G):
    """A spread of small graphs: empty, edge, path, triangle, K5, two K4
    sharing an edge, a star, isolated vertices, random ones with planted cliques."""
    out = [
        G.from_edges(1, [], "single"),
        G.from_edges(5, [], "no-edges"),
        G.from_edges(2, [(0, 1)], "edge"),
        G.from_edges(4, [(0, 1), (1, 2), (2, 3)], "path4"),
        G.from_edges(3, [(0, 1), (1, 2), (0, 2)], "triangle"),
        G.from_edges(5, [(a, b) for a in range(5) for b in range(a + 1, 5)], "K5"),
        G.from_edges(6, [(0, 1), (0, 2), (0, 3), (1, 2), (1, 3), (2, 3), (2, 4), (3, 4), (2, 5), (3, 5), (4, 5)],
                     "two-K4"),
        G.from_edges(7, [(0, i) for i in range(1, 7)], "star"),
        G.from_edges(8, [(1, 2), (2, 3), (1, 3), (5, 6)], "isolated+tri"),
        G.from_edges(4, [(0, 1), (1, 2), (2, 3), (3, 0)], "C4"),
    ]
    for s in range(6):
        out.append(random_graph(G, 30 + 5 * s, 0.15 + 0.05 * s, 100 + s, planted=[tuple(range(s, s + 6))]))
    out.append(random_graph(G, 60, 0.3, 999, planted=[tuple(range(0, 40, 3)), tuple(range(1, 50, 4))]))
    return out
