"""The CPU oracle against closed forms, brute force and the textbook search."""
import os
import numpy as np
import pytest

import mce_b200 as mce
import oracle
from graphs import KNOWN


def hist_dict(h):
    return {int(i): int(h[i]) for i in np.nonzero(h)[0]}


@pytest.mark.parametrize("name,make,total,sizes", KNOWN, ids=[k[0] for k in KNOWN])
def test_oracle_known_answers(name, make, total, sizes):
    g = make()
    t, h, _ = oracle.count(g)
    assert t == total
    assert hist_dict(h) == sizes
    t2, h2 = oracle.tomita(g)
    assert (t2, hist_dict(h2)) == (total, sizes)
    if g.n <= 22:  # brute force visits every clique: 2^n for K_n
        t3, h3 = oracle.brute(g)
        assert (t3, hist_dict(h3)) == (total, sizes)


@pytest.mark.parametrize("seed", range(40))
def test_oracle_vs_brute_random(seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(2, 24))
    p = float(rng.uniform(0.1, 0.9))
    iu = np.triu_indices(n, 1)
    keep = rng.random(len(iu[0])) < p
    g = mce.from_edges(iu[0][keep], iu[1][keep], n)
    t, h, _ = oracle.count(g)
    tb, hb = oracle.brute(g)
    assert t == tb
    assert np.array_equal(h, hb)


@pytest.mark.parametrize("seed", range(6))
def test_oracle_vs_tomita_medium(seed):
    g = mce.gen_er(300, 0.08, seed, planted=4, cmin=5, cmax=15)
    t, h, _ = oracle.count(g)
    tt, ht = oracle.tomita(g)
    assert t == tt and np.array_equal(h, ht)


def test_peel_invariants():
    """Core numbers and the orientation bound d+(v) <= core(v)."""
    g = mce.gen_rmat(10, 16, 0.57, 0.19, 0.19, 7)
    prio, core, dg = oracle.peel(g)
    deg = np.diff(g.row_ptr[:g.n + 1])
    assert dg == core.max()
    # core number: v has at least core(v) neighbours of core >= core(v)
    for v in range(g.n):
        nb = g.col[g.row_ptr[v]:g.row_ptr[v + 1]]
        assert np.count_nonzero(core[nb] >= core[v]) >= core[v]
    split, cs = oracle.orient(g, prio)
    dplus = g.row_ptr[1:g.n + 1] - split
    assert np.all(dplus <= core)
    assert np.all(deg >= 0)
    # the final round keeps priority m and is the maximal core
    last = prio == g.m
    assert last.any() and np.all(core[last] == dg)


def test_peel_round_numbering_small():
    """Path 0-1-2-3-4: level 1 rounds {0,4} then {1,3}; vertex 2 is the last round."""
    from graphs import path
    g = path(5)
    prio, core, dg = oracle.peel(g)
    assert list(prio) == [0, 1, g.m, 1, 0]
    assert list(core) == [1, 1, 1, 1, 1] and dg == 1


def test_isolated_vertices_not_counted():
    from graphs import build
    g = build(6, [(0, 1)])  # 4 isolated vertices + one edge
    assert oracle.count(g)[0] == 1


def test_per_root_sum_equals_total():
    g = mce.gen_er(2000, 0.01, 5, planted=10, cmin=6, cmax=14)
    tot, h, rc, rn = oracle.roots(g)
    assert rc.sum() == tot == oracle.count(g)[0]
    assert np.all(rn[rc > 0] > 0)


def test_workload_generators_match_the_library():
    """The checker's second build of the seeded generators (used where
    libmce.so must not be loaded, e.g. bench.py's reference arm) returns the
    library's graphs byte for byte, and its .bel file is the library's."""
    import tempfile
    b = mce.gen_chung_lu_batch(64, 64, 2048, 2.3, 8.0, 32.0, 5, 5, 40, 11)
    u = mce.union(b)
    ou, start = oracle.gen_batch_union(64, 64, 2048, 2.3, 8.0, 32.0, 5, 5, 40, 11)
    assert np.array_equal(ou.row_ptr, u.row_ptr[:u.n + 1]) and np.array_equal(ou.col, u.col)
    assert np.array_equal(start, b.vtx_offsets - np.arange(65))
    for og, lg in ((oracle.gen_ba(20000, 8, 23, 20, 20, 60), mce.gen_ba(20000, 8, 23, 20, 20, 60)),
                   (oracle.gen_rmat(10, 16, 0.57, 0.19, 0.19, 7),
                    mce.gen_rmat(10, 16, 0.57, 0.19, 0.19, 7)),
                   (oracle.gen_er(3000, 0.004, 1, 5, 6, 12), mce.gen_er(3000, 0.004, 1, 5, 6, 12))):
        assert np.array_equal(og.row_ptr, lg.row_ptr[:lg.n + 1]) and np.array_equal(og.col, lg.col)
    with tempfile.TemporaryDirectory() as d:
        oracle.bel_write(os.path.join(d, "a.bel"), ou)
        mce.bel_write(os.path.join(d, "b.bel"), u)
        with open(os.path.join(d, "a.bel"), "rb") as fa, open(os.path.join(d, "b.bel"), "rb") as fb:
            assert fa.read() == fb.read()
    # per-graph sums of per-root counts equal each graph's own count
    _, _, rc, _ = oracle.roots(ou)
    per = oracle.per_graph(rc, start)
    for i in (0, 7, 63):
        assert int(per[i]) == oracle.count(b.graph(i))[0]
