"""CUDA path vs the CPU oracle: bit-exact counts, histograms, orders and trees."""
import os
import subprocess

import numpy as np
import pytest

import mce_b200 as mce
import oracle
from graphs import KNOWN, build

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "mce-gpu_b200", "bin", "parallel_mce_on_gpus")


def gpu_count(g, **kw):
    with mce.Graph.from_host(g) as dg:
        return dg.count(**kw)


def assert_same(g, **kw):
    r = gpu_count(g, **kw)
    t, h, dg = oracle.count(g)
    assert r.total == t, (r.total, t)
    assert np.array_equal(r.hist, h)
    assert r.stats["error_flags"] == 0
    return r


@pytest.mark.parametrize("name,make,total,sizes", KNOWN, ids=[k[0] for k in KNOWN])
def test_known_answers(name, make, total, sizes):
    r = gpu_count(make())
    assert r.total == total
    assert {int(i): int(r.hist[i]) for i in np.nonzero(r.hist)[0]} == sizes


@pytest.mark.parametrize("seed", range(12))
@pytest.mark.parametrize("width", [32, 64])
def test_random_small(seed, width):
    rng = np.random.default_rng(1000 + seed)
    n = int(rng.integers(5, 400))
    p = float(rng.uniform(0.01, 0.5))
    g = mce.gen_er(n, p, seed, planted=int(rng.integers(0, 4)), cmin=4, cmax=min(n, 30))
    assert_same(g, bitmap_width=width)


def test_small_plain_config():
    """ER(10000, 0.002), seed 1, + 20 planted cliques of size 6..12, 32-bit rows."""
    g = mce.gen_er(10000, 0.002, 1, 20, 6, 12)
    r = assert_same(g, bitmap_width=32)
    assert r.total == 97157  # the reference binary prints the same count (tests/golden)


def hubs_graph(n, hubs, seed):
    """ER(n, 4/n) plus the given vertices adjacent to every other vertex:
    rows of n - 1 arcs among many short ones."""
    base = mce.gen_er(n, 4.0 / n, seed)
    edges = {(v, int(w)) for v in range(base.n)
             for w in base.col[base.row_ptr[v]:base.row_ptr[v + 1]] if v < w}
    for h in hubs:
        edges |= {(min(h, v), max(h, v)) for v in range(n) if v != h}
    return build(n, sorted(edges))


@pytest.mark.parametrize("maker", [
    lambda: mce.gen_er(3000, 0.01, 3, 10, 6, 20),
    lambda: mce.gen_rmat(11, 16, 0.57, 0.19, 0.19, 7),
    lambda: mce.gen_ba(20000, 8, 5, 20, 20, 60),
    lambda: build(5, [(0, 1), (1, 2), (2, 3), (3, 4)]),
    # rows longer than 2,048 arcs: split by a whole block, after the rest
    lambda: mce.gen_rmat(14, 16, 0.57, 0.19, 0.19, 7),
    lambda: hubs_graph(12000, [0, 5, 77], 3),
])
def test_degeneracy_bit_exact(maker):
    g = maker()
    prio_o, core_o, dg_o = oracle.peel(g)
    with mce.Graph.from_host(g) as dg:
        prio, core, d = dg.degeneracy()
        assert d == dg_o
        assert np.array_equal(core, core_o)
        assert np.array_equal(prio, prio_o)
        split, cs = dg.split_csr()
    split_o, cs_o = oracle.orient(g, prio_o)
    assert np.array_equal(split, split_o)
    assert np.array_equal(cs, cs_o)


@pytest.mark.parametrize("maker", [
    lambda: mce.gen_er(4000, 0.01, 9, 12, 8, 40),
    lambda: mce.gen_rmat(11, 16, 0.57, 0.19, 0.19, 7),
])
def test_per_root_counts_and_tree_sizes(maker):
    g = maker()
    tot, h, rc_o, rn_o = oracle.roots(g)
    with mce.Graph.from_host(g) as dg:
        r = dg.count(log_roots=True)
        rc, rn = dg.root_counts(), dg.root_log()
    assert r.total == tot
    assert np.array_equal(rc, rc_o)
    assert np.array_equal(rn, rn_o)  # same pivot rule and tie-break -> same trees
    assert r.stats["tree_nodes"] == int(rn_o.sum())


def test_rmat_scale13_wide_roots():
    """R-MAT (0.57,0.19,0.19,0.05) scale 13: later degrees up to 90 (wide engine)."""
    g = mce.gen_rmat(13, 16, 0.57, 0.19, 0.19, 7)
    r = assert_same(g)
    assert r.stats["class_roots"][2] > 0  # wide-engine roots exercised


@pytest.mark.parametrize("n", [5000, 18000])
def test_hub_with_many_earlier_neighbours(n):
    """Vertex 0 is adjacent to every vertex and sits in a K8 on 0..7, which
    is peeled last (the sparse rest has a smaller core): its earlier list
    holds n - 8 vertices, its later list 7.  Up to 16,384 earlier neighbours
    such a root stays in a register engine (whose slab grows to a power of
    two covering them); beyond that it lands in the wide engine."""
    base = mce.gen_er(n, 6.0 / n, 11)
    s, d = [], []
    for v in range(base.n):
        for w in base.col[base.row_ptr[v]:base.row_ptr[v + 1]]:
            if v < w:
                s.append(v); d.append(int(w))
    s += [0] * (n - 1)
    d += list(range(1, n))
    for v in range(1, 8):
        for w in range(v + 1, 8):
            s.append(v); d.append(w)
    g = mce.from_edges(np.array(s), np.array(d), n)
    r = assert_same(g)
    assert r.stats["class_roots"][2] == (0 if n - 8 <= 16384 else 1)


def test_cliques_wider_than_64():
    """Planted cliques of 70..300 vertices: roots with d+ up to 299."""
    g = mce.gen_er(2000, 0.005, 21, 6, 70, 300)
    assert_same(g)


def test_ba_with_planted_cliques():
    g = mce.gen_ba(100000, 8, 23, 40, 20, 60)
    assert_same(g)


def test_chung_lu_batch_union():
    b = mce.gen_chung_lu_batch(48, 64, 16384, 2.3, 8, 32, 5, 5, 40, 11)
    assert_same(mce.union(b))


def test_permutation_invariance():
    g = mce.gen_rmat(12, 16, 0.57, 0.19, 0.19, 3)
    a = gpu_count(g)
    b = gpu_count(mce.permute(g, 5))
    assert a.total == b.total and np.array_equal(a.hist, b.hist)


def test_degenerate_graphs():
    assert gpu_count(build(10, [])).total == 0
    assert gpu_count(build(2, [(0, 1)])).total == 1
    g = mce.HostGraph(np.zeros(1, np.int32), np.zeros(0, np.int32), 0, 0)
    assert gpu_count(g).total == 0


def test_repeated_calls_identical():
    g = mce.gen_ba(50000, 6, 1, 10, 10, 30)
    with mce.Graph.from_host(g) as dg:
        a = dg.count()
        b = dg.count(bitmap_width=64)
        c = dg.count()
    assert a.total == b.total == c.total
    assert np.array_equal(a.hist, c.hist) and np.array_equal(a.hist, b.hist)


def test_cli_matches_oracle(tmp_path):
    g = mce.gen_er(3000, 0.01, 4, 8, 6, 16)
    bel = str(tmp_path / "g.bel")
    mce.bel_write(bel, g)
    r = subprocess.run([CLI, "-m", "mce", "-g", bel, "-d", "0", "-p", "l1", "-i", "p", "-w", "wl"],
                       capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    t, _, dgn = oracle.count(g)
    assert f"Found {t} maximal cliques in total." in r.stdout
    assert f"Max Core = {dgn}" in r.stdout
    assert "Degeneracy ordering time:" in r.stdout and "count time" in r.stdout


def _hub_over(g_inner, extra=3):
    """g_inner plus `extra` hubs adjacent to every vertex: the hubs' trees are
    the whole search of g_inner, so they are split among warps."""
    s, d = [], []
    n = g_inner.n
    for v in range(n):
        for w in g_inner.col[g_inner.row_ptr[v]:g_inner.row_ptr[v + 1]]:
            if v < w:
                s.append(v); d.append(int(w))
    for h in range(extra):
        for v in range(n):
            s.append(n + h); d.append(v)
    return mce.from_edges(np.array(s), np.array(d), n + extra)


@pytest.mark.parametrize("maker", [
    lambda: mce.gen_rmat(12, 16, 0.57, 0.19, 0.19, 7),
    lambda: _hub_over(__import__("graphs").moon_moser(9)),      # 3^9 cliques under the hubs
    lambda: _hub_over(mce.gen_er(60, 0.5, 3)),                   # 60 later neighbours: 64-bit engine
    lambda: _hub_over(mce.gen_er(120, 0.45, 4), extra=2),        # wide engine
])
def test_worker_list_on_off_identical(maker):
    g = maker()
    t, h, rc_o, rn_o = oracle.roots(g)
    out = {}
    with mce.Graph.from_host(g) as dg:
        # (sharing, smallest shared candidate set, nodes walked before sharing)
        for wl, dmin, after in ((mce.WL_ON, 2, 1), (mce.WL_ON, 10, 1), (mce.WL_ON, 10, 0),
                                (mce.WL_OFF, 10, 0)):
            r = dg.count(worker_list=wl, donate_threshold=dmin, donate_after=after, log_roots=True)
            out[(wl, dmin, after)] = (r.total, r.hist.copy(), dg.root_counts(), dg.root_log())
            if wl == mce.WL_ON and after == 1:
                assert r.stats["donations"] > 0  # the sharing path really ran
    for (tot, hist, rc, rn) in out.values():
        assert tot == t and np.array_equal(hist, h)
        assert np.array_equal(rc, rc_o)
        assert np.array_equal(rn, rn_o)  # donation moves subtrees, never changes them


def test_warp_log_accounts_for_every_node_and_donation():
    hg = mce.gen_rmat(12, 16, 0.57, 0.19, 0.19, 7)
    with mce.Graph.from_host(hg) as g:
        r = g.count(warp_log=True, donate_after=1)
        log = g.warp_log()
        plain = g.count()
    assert r.total == plain.total
    assert len(log["sm"]) > 0 and int(log["sm"].max()) < 1024
    assert int(log["nodes"].sum()) == r.stats["tree_nodes"]
    assert int(log["donations"].sum()) == r.stats["donations"] and r.stats["donations"] > 0


def test_warp_cycle_breakdown():
    hg = mce.gen_rmat(12, 16, 0.57, 0.19, 0.19, 7)
    with mce.Graph.from_host(hg) as g:
        r = g.count(warp_log=2)
        log = g.warp_log()
    assert r.total == oracle.count(hg)[0]
    cyc = log["cycles"].astype(np.float64)
    assert cyc.shape == (len(log["sm"]), 7)
    busy = cyc.sum(axis=0)
    # every warp encodes, pivots, branches and tests leaves
    assert busy[1] > 0 and busy[3] > 0 and busy[5] > 0 and busy[6] > 0
    assert int(log["nodes"].sum()) == r.stats["tree_nodes"]


@pytest.mark.skipif(not os.path.exists(CLI), reason="CLI not built")
@pytest.mark.parametrize("task,header", [("mce-lb-eval", "Number of traversed nodes"),
                                         ("mce-donor-eval", "Number of donations"),
                                         ("mce-bd-eval", "TESTING MAXIMALITY")])
def test_cli_eval_lines(tmp_path, task, header):
    import re
    import subprocess
    hg = mce.gen_rmat(11, 16, 0.57, 0.19, 0.19, 7)
    bel = str(tmp_path / "g.bel")
    mce.bel_write(bel, hg)
    out = subprocess.run([CLI, "-m", task, "-g", bel, "-d", "0", "-p", "l1", "-i", "p", "-w", "wl"],
                         capture_output=True, text=True, timeout=120).stdout
    assert header in out
    found = int(re.findall(r"Found (.*) maximal cliques in total", out)[0].replace(",", ""))
    assert found == oracle.count(hg)[0]
    if task == "mce-bd-eval":  # plot.py's parse_mce_bd pattern: seven columns
        rows = re.findall(r"([0-9]+)" + r", ([0-9]+)" * 6, out)
        assert len(rows) > 0 and sum(int(x) for row in rows for x in row) > 0
    else:  # plot.py's parse_mce_lb pattern
        rows = re.findall(r"([0-9]+), ([0-9]+), ([0-9]+)", out)
        assert len(rows) > 0 and all(int(sm) < 1024 for _, sm, _ in rows)


@pytest.mark.parametrize("wide_blocks", [4, 8])
def test_wide_engine_occupancy_variants(wide_blocks):
    g = mce.gen_er(2000, 0.005, 21, planted=6, cmin=70, cmax=300)  # roots in the wide engine
    t, h, _ = oracle.count(g)
    with mce.Graph.from_host(g) as dg:
        r = dg.count(wide_blocks=wide_blocks, log_roots=True)
        nodes = dg.root_log()
    assert r.stats["class_roots"][2] > 0
    assert r.total == t and np.array_equal(r.hist, h)
    assert np.array_equal(nodes, oracle.roots(g)[3])


@pytest.mark.parametrize("maker", [
    lambda: mce.gen_er(2000, 0.01, 1, 8, 6, 40),            # all three engines
    lambda: mce.gen_rmat(12, 16, 0.57, 0.19, 0.19, 7),      # wide roots
    lambda: mce.gen_ba(20000, 8, 5, 20, 20, 60),            # 64-bit rows, long lists
    lambda: _hub_graph(5000),                               # hub rows
    lambda: mce.union(mce.gen_chung_lu_batch(32, 64, 4096, 2.3, 8, 32, 5, 5, 40, 13)),
], ids=["er", "rmat12", "ba", "hub", "batch"])
@pytest.mark.parametrize("kw", [{}, {"worker_list": mce.WL_OFF}, {"bitmap_width": 64},
                                {"cuda_graph": 1}], ids=["wl", "nowl", "64bit", "graph"])
def test_level2_edge_rooted_units(maker, kw):
    """-p l2: every oriented edge (r, v) is a unit (the triangle list as its
    candidates, its pivot from them alone, the root's neighbours before v
    outside): counts, histogram and per-root counts are those of L1, and the
    per-root tree sizes those of the oracle's L2 walk (units are not nodes)."""
    g = maker()
    t, h, rc, rn = oracle.roots_l2(g)
    with mce.Graph.from_host(g) as dg:
        for _ in range(2):
            r = dg.count(level=mce.LEVEL_L2, log_roots=True, **kw)
            assert r.stats["error_flags"] == 0
            assert r.total == t and np.array_equal(r.hist, h)
            assert np.array_equal(dg.root_counts(), rc)
            assert np.array_equal(dg.root_log(), rn)
    assert t == oracle.count(g)[0]


def test_level2_lists_the_same_cliques():
    g = mce.gen_er(600, 0.03, 2, 6, 5, 14)
    with mce.Graph.from_host(g) as dg:
        l1 = sorted(tuple(sorted(c)) for c in dg.list_cliques())
        l2 = sorted(tuple(sorted(c)) for c in dg.list_cliques(level=mce.LEVEL_L2))
    assert l1 == l2


def test_level2_on_a_batch():
    b = mce.gen_chung_lu_batch(48, 64, 4096, 2.3, 8, 32, 5, 5, 40, 17)
    per_o = [oracle.count(b.graph(i))[0] for i in range(b.num_graphs)]
    with mce.Batch(b) as db:
        r = db.count(level=mce.LEVEL_L2)
    assert [int(x) for x in r.per_graph] == per_o


@pytest.mark.parametrize("maker", [
    lambda: mce.gen_rmat(12, 16, 0.57, 0.19, 0.19, 7),
    lambda: mce.gen_ba(40000, 8, 9, 20, 20, 60),
    lambda: mce.union(mce.gen_chung_lu_batch(32, 64, 4096, 2.3, 8, 32, 5, 5, 40, 13)),
])
def test_x_pivot_changes_trees_not_counts(maker):
    g = maker()
    t, h, _ = oracle.count(g)
    _, _, rc, _ = oracle.roots(g)
    with mce.Graph.from_host(g) as dg:
        ip = dg.count()
        px = dg.count(induced=mce.INDUCED_PX, log_roots=True)
        counts = dg.root_counts()
    assert px.total == t and np.array_equal(px.hist, h)
    assert np.array_equal(counts, rc)  # a root's cliques do not depend on its pivots
    assert px.stats["tree_nodes"] <= ip.stats["tree_nodes"]


@pytest.mark.parametrize("kw", [{}, {"worker_list": mce.WL_OFF}, {"wide_blocks": 8},
                                {"warps_per_root": 2}, {"level": mce.LEVEL_L2}],
                         ids=["wl", "nowl", "wide8", "w2", "l2"])
def test_x_pivot_in_the_wide_engine(kw):
    """-i px in the wide engine (roots with more than 64 later neighbours):
    the same counts and per-root counts, no more tree nodes in its class."""
    g = mce.gen_rmat(13, 16, 0.57, 0.19, 0.19, 7)
    t, h, _ = oracle.count(g)
    _, _, rc, _ = oracle.roots(g)
    with mce.Graph.from_host(g) as dg:
        ip = dg.count(log_roots=True, **kw)
        n_ip = dg.root_log()
        px = dg.count(x_pivot=1, log_roots=True, **kw)
        counts, n_px = dg.root_counts(), dg.root_log()
        split, _ = dg.split_csr()
    assert px.stats["class_roots"][2] > 0 and px.stats["error_flags"] == 0
    assert px.total == t and np.array_equal(px.hist, h)
    assert np.array_equal(counts, rc)
    wide = (g.row_ptr[1:g.n + 1] - split) > 64
    assert n_px[wide].sum() <= n_ip[wide].sum()  # the outside pivots prune wide trees
    if not kw:
        assert n_px[wide].sum() < n_ip[wide].sum()


@pytest.mark.parametrize("maker,kw", [
    (lambda: mce.gen_er(2000, 0.01, 1, 8, 6, 40), {}),                    # all three engines
    (lambda: mce.gen_er(2000, 0.01, 1, 8, 6, 40), {"bitmap_width": 64}),
    (lambda: mce.gen_er(2000, 0.01, 1, 8, 6, 40), {"worker_list": mce.WL_OFF}),
    (lambda: mce.gen_rmat(12, 16, 0.57, 0.19, 0.19, 7), {"donate_after": 16}),  # wide roots, tasks
    (lambda: mce.gen_ba(20000, 8, 5, 20, 20, 60), {}),
])
def test_word_ops_per_root_equal_the_oracle(maker, kw):
    """opts.count_ops: the search's algorithmic 32-bit word operations (2 W
    per row scored by a pivot selection + 4 W per tree node, W = ceil(d+/32))
    equal the oracle's walk root by root, with subtrees shared or not, and
    the counting variants give the same counts and trees."""
    g = maker()
    tot, rc_o, rn_o, ro_o = oracle.roots_ops(g)
    with mce.Graph.from_host(g) as dg:
        r = dg.count(log_roots=True, count_ops=True, **kw)
        rc, rn, ro = dg.root_counts(), dg.root_log(), dg.root_ops()
        plain = dg.count(**kw)
    assert r.total == tot == plain.total
    assert np.array_equal(rc, rc_o) and np.array_equal(rn, rn_o)
    assert np.array_equal(ro, ro_o)
    assert r.stats["word_ops"] == int(ro_o.sum()) > 0
    assert plain.stats["word_ops"] == 0
    assert r.stats["tree_nodes"] == plain.stats["tree_nodes"]


def test_word_ops_on_a_batch():
    b = mce.gen_chung_lu_batch(32, 64, 2048, 2.3, 8, 32, 3, 5, 30, 5)
    u = mce.union(b)
    _, _, _, ro_o = oracle.roots_ops(u)
    with mce.Batch(b) as db:
        r = db.count(count_ops=True)
    assert r.stats["word_ops"] == int(ro_o.sum())


def test_word_ops_rejects_other_modes():
    g = mce.gen_er(500, 0.02, 1)
    with mce.Graph.from_host(g) as dg:
        for kw in ({"x_pivot": 1}, {"warp_log": 1}):
            with pytest.raises(mce.MceError) as e:
                dg.count(count_ops=True, **kw)
            assert e.value.code == mce.EINVAL


def _hub_graph(n):
    """Vertex 0 adjacent to every vertex and in a K8 on 0..7 that is peeled
    last: a root with n - 8 earlier neighbours (a hub) and 7 later ones."""
    base = mce.gen_er(n, 6.0 / n, 11)
    s, d = [], []
    for v in range(base.n):
        for w in base.col[base.row_ptr[v]:base.row_ptr[v + 1]]:
            if v < w:
                s.append(v); d.append(int(w))
    s += [0] * (n - 1)
    d += list(range(1, n))
    for v in range(1, 8):
        for w in range(v + 1, 8):
            s.append(v); d.append(w)
    return mce.from_edges(np.array(s), np.array(d), n)


@pytest.mark.parametrize("maker", [
    lambda: mce.gen_er(2000, 0.01, 1, 8, 6, 40),                  # all three engines
    lambda: mce.gen_rmat(12, 16, 0.57, 0.19, 0.19, 7),            # wide roots and tasks
    lambda: _hub_graph(5000),                                      # a hub root split in parts
], ids=["er", "rmat12", "hub"])
@pytest.mark.parametrize("kw", [
    {"warps_per_root": 2}, {"warps_per_root": 4},
    {"bucket_warps_per_root": (3, 2, 4), "bucket_donate_threshold": (6, 16, 8),
     "bucket_donate_after": (64, 1024, 16)},
    {"warps_per_root": 3, "worker_list": mce.WL_OFF},
    {"warps_per_root": 2, "bitmap_width": 64, "cuda_graph": 1},
], ids=["w2", "w4", "buckets", "w3-nowl", "w2-64bit-graph"])
def test_warps_per_root_give_the_same_trees(maker, kw):
    """Several warps per root split a root's tree by its first-level
    branches: per-root counts and tree sizes stay the oracle's, and the
    histogram the whole graph's."""
    g = maker()
    tot, h, rc_o, rn_o = oracle.roots(g)
    with mce.Graph.from_host(g) as dg:
        for _ in range(2):  # also a second call (a replayed capture with cuda_graph)
            r = dg.count(log_roots=True, **kw)
            assert r.stats["error_flags"] == 0
            assert r.total == tot and np.array_equal(r.hist, h)
            assert np.array_equal(dg.root_counts(), rc_o)
            assert np.array_equal(dg.root_log(), rn_o)


def test_warps_per_root_word_ops():
    g = mce.gen_er(2000, 0.01, 1, 8, 6, 40)
    _, _, _, ro_o = oracle.roots_ops(g)
    with mce.Graph.from_host(g) as dg:
        r = dg.count(count_ops=True, log_roots=True, warps_per_root=3)
        assert np.array_equal(dg.root_ops(), ro_o)
    assert r.stats["word_ops"] == int(ro_o.sum())


def test_per_bucket_settings_on_a_batch():
    b = mce.gen_chung_lu_batch(48, 64, 4096, 2.3, 8, 32, 5, 5, 40, 21)
    per_o = [oracle.count(b.graph(i))[0] for i in range(b.num_graphs)]
    with mce.Batch(b) as db:
        for kw in ({}, {"bucket_warps_per_root": (1, 4, 2), "bucket_donate_threshold": (8, 6, 0)}):
            r = db.count(**kw)
            assert [int(x) for x in r.per_graph] == per_o


def test_warps_per_root_bounds():
    g = mce.gen_er(300, 0.05, 1)
    with mce.Graph.from_host(g) as dg:
        for kw in ({"warps_per_root": 33}, {"warps_per_root": -1},
                   {"bucket_warps_per_root": (0, 40, 0)}):
            with pytest.raises(mce.MceError) as e:
                dg.count(**kw)
            assert e.value.code == mce.EINVAL


@pytest.mark.parametrize("maker", [
    lambda: mce.gen_er(2000, 0.01, 1, 8, 6, 40),            # small and large roots
    lambda: mce.gen_ba(20000, 8, 5, 20, 20, 60),            # lists too long to stage together
    lambda: _hub_graph(5000),                               # hub rows
    lambda: build(4, [(0, 1), (1, 2), (2, 3), (0, 3), (0, 2)]),  # lists ending at the last arc
    lambda: mce.gen_er(3, 1.0, 1),
], ids=["er", "ba", "hub", "tail", "k3"])
def test_staged_lists_give_the_same_trees(maker):
    """opts.stage_lists: the 32-bit engine copies the lists it encodes into
    shared memory with 1-D bulk copies; counts and per-root trees stay the
    oracle's."""
    g = maker()
    tot, h, rc_o, rn_o = oracle.roots(g)
    with mce.Graph.from_host(g) as dg:
        for _ in range(2):
            r = dg.count(log_roots=True, stage_lists=1)
            assert r.stats["error_flags"] == 0
            assert r.total == tot and np.array_equal(r.hist, h)
            assert np.array_equal(dg.root_counts(), rc_o) and np.array_equal(dg.root_log(), rn_o)


def test_staged_lists_on_a_batch():
    b = mce.gen_chung_lu_batch(64, 64, 4096, 2.3, 8, 32, 5, 5, 40, 13)
    per_o = [oracle.count(b.graph(i))[0] for i in range(b.num_graphs)]
    with mce.Batch(b) as db:
        for _ in range(2):
            r = db.count(stage_lists=1)
            assert [int(x) for x in r.per_graph] == per_o
