"""Clique listing (mce_list) against a pure-Python Tomita enumeration."""
import numpy as np
import pytest

import mce_b200 as mce
import oracle
from graphs import KNOWN

pytestmark = pytest.mark.gpu


def python_cliques(g):
    """Every maximal clique of size >= 2 (Bron-Kerbosch with Tomita pivoting)."""
    adj = [set(int(w) for w in g.col[g.row_ptr[v]:g.row_ptr[v + 1]]) for v in range(g.n)]
    out = []

    def bk(R, P, X):
        if not P and not X:
            if len(R) >= 2:
                out.append(frozenset(R))
            return
        u = max(P | X, key=lambda w: len(P & adj[w]))
        for v in list(P - adj[u]):
            bk(R | {v}, P & adj[v], X & adj[v])
            P = P - {v}
            X = X | {v}

    bk(set(), set(range(g.n)), set())
    return out


def check(g, **opts):
    with mce.Graph.from_host(g) as dg:
        got = dg.list_cliques(**opts)
        total = dg.count().total
    sets = [frozenset(int(x) for x in c) for c in got]
    assert len(sets) == total == len(set(sets))
    assert set(sets) == set(python_cliques(g))
    return got


@pytest.mark.parametrize("name,make,total,sizes", KNOWN, ids=[k[0] for k in KNOWN])
def test_list_known_graphs(name, make, total, sizes):
    assert len(check(make())) == total


@pytest.mark.parametrize("maker", [
    lambda: mce.gen_er(80, 0.15, 4),
    lambda: mce.gen_rmat(8, 8, 0.57, 0.19, 0.19, 7),
    lambda: mce.gen_er(400, 0.02, 3, planted=3, cmin=70, cmax=90),  # wide roots
])
def test_list_matches_enumeration(maker):
    got = check(maker())
    for c in got:  # the root is the clique's first member, the rest ascending
        assert list(c[1:]) == sorted(c[1:])


def test_list_grows_buffers_and_shares_subtrees():
    g = mce.gen_rmat(10, 16, 0.57, 0.19, 0.19, 7)
    with mce.Graph.from_host(g) as dg:
        got = dg.list_cliques(ids_cap=16, cliques_cap=4, donate_after=1)
    assert len(got) == oracle.count(g)[0]
    sizes = np.bincount([len(c) for c in got], minlength=mce.HIST_MAX)
    assert np.array_equal(sizes, oracle.count(g)[1])
