"""Closed-form graphs with known maximal-clique counts (size >= 2)."""
import itertools

import numpy as np

import mce_b200 as mce


def build(n, edges):
    if edges:
        s, d = zip(*edges)
    else:
        s, d = (), ()
    return mce.from_edges(np.array(s, np.int64), np.array(d, np.int64), n)


def complete(n):
    return build(n, list(itertools.combinations(range(n), 2)))


def cycle(n):
    return build(n, [(i, (i + 1) % n) for i in range(n)])


def path(n):
    return build(n, [(i, i + 1) for i in range(n - 1)])


def star(k):
    return build(k + 1, [(0, i) for i in range(1, k + 1)])


def multipartite(parts):
    """Complete multipartite graph: prod(parts) maximal cliques of size len(parts)."""
    ids, base = [], 0
    for p in parts:
        ids.append(list(range(base, base + p)))
        base += p
    edges = [(u, v) for a, b in itertools.combinations(range(len(parts)), 2)
             for u in ids[a] for v in ids[b]]
    return build(base, edges)


def moon_moser(k):
    return multipartite([3] * k)


def disjoint_cliques(sizes):
    edges, base = [], 0
    for s in sizes:
        edges += [(base + a, base + b) for a, b in itertools.combinations(range(s), 2)]
        base += s
    return build(base, edges)


def wheel(n):
    return build(n + 1, [(0, i) for i in range(1, n + 1)] +
                 [(i, i % n + 1) for i in range(1, n + 1)])


def petersen():
    outer = [(i, (i + 1) % 5) for i in range(5)]
    spokes = [(i, i + 5) for i in range(5)]
    inner = [(5 + i, 5 + (i + 2) % 5) for i in range(5)]
    return build(10, outer + spokes + inner)


def empty(n):
    return build(n, [])


# (name, graph factory, expected total, expected {size: count})
KNOWN = [
    ("K2", lambda: complete(2), 1, {2: 1}),
    ("K7", lambda: complete(7), 1, {7: 1}),
    ("K33", lambda: complete(33), 1, {33: 1}),
    ("K64", lambda: complete(64), 1, {64: 1}),
    ("K65", lambda: complete(65), 1, {65: 1}),
    ("C3", lambda: cycle(3), 1, {3: 1}),
    ("C4", lambda: cycle(4), 4, {2: 4}),
    ("C50", lambda: cycle(50), 50, {2: 50}),
    ("P10", lambda: path(10), 9, {2: 9}),
    ("star40", lambda: star(40), 40, {2: 40}),
    ("K_5_7", lambda: multipartite([5, 7]), 35, {2: 35}),
    ("moon_moser_4", lambda: moon_moser(4), 81, {4: 81}),
    ("moon_moser_8", lambda: moon_moser(8), 6561, {8: 6561}),
    ("turan_2345", lambda: multipartite([2, 3, 4, 5]), 120, {4: 120}),
    ("cliques_3_5_9", lambda: disjoint_cliques([3, 5, 9, 1]), 3, {3: 1, 5: 1, 9: 1}),
    ("wheel9", lambda: wheel(9), 9, {3: 9}),
    ("petersen", petersen, 15, {2: 15}),
    ("empty50", lambda: empty(50), 0, {}),
]
