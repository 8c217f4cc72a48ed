"""Batched counting (mce_batch_*): per-graph counts against the oracle."""
import numpy as np
import pytest

import mce_b200 as mce
import oracle

pytestmark = pytest.mark.gpu


def per_graph_oracle(b):
    return np.array([oracle.count(b.graph(i))[0] for i in range(b.num_graphs)], np.uint64)


def test_batch_per_graph_counts_exact():
    b = mce.gen_chung_lu_batch(96, 64, 4096, 2.3, 8, 32, 5, 5, 40, 11)
    want = per_graph_oracle(b)
    _, h_union, _ = oracle.count(mce.union(b))
    with mce.Batch(b) as db:
        r = db.count()
        r2 = db.count()  # replay of the captured search launches
    assert np.array_equal(r.per_graph, want)
    assert r.total == int(want.sum()) and np.array_equal(r.hist, h_union)
    assert np.array_equal(r2.per_graph, want) and np.array_equal(r2.hist, r.hist)


def test_batch_graph_mode_and_plain_mode_agree():
    b = mce.gen_chung_lu_batch(40, 64, 2048, 2.3, 8, 32, 5, 5, 40, 7)
    with mce.Batch(b) as db:
        a = db.count(cuda_graph=1)
        p = db.count(cuda_graph=0)
        w = db.count(cuda_graph=1, worker_list=mce.WL_OFF)
    assert np.array_equal(a.per_graph, p.per_graph) and np.array_equal(a.per_graph, w.per_graph)


def test_batch_reload_smaller_and_larger():
    b1 = mce.gen_chung_lu_batch(32, 64, 2048, 2.3, 8, 32, 5, 5, 40, 1)
    b2 = mce.gen_chung_lu_batch(8, 64, 1024, 2.3, 8, 32, 5, 5, 40, 2)
    b3 = mce.gen_chung_lu_batch(64, 64, 4096, 2.3, 8, 32, 5, 5, 40, 3)
    with mce.Batch(b1) as db:
        assert np.array_equal(db.count().per_graph, per_graph_oracle(b1))
        for b in (b2, b3, b1):
            rp, col, vo, ao = mce.Batch._arrays(b)
            db.reload_ptr(rp.ctypes.data, col.ctypes.data, vo.ctypes.data, ao.ctypes.data,
                          b.num_graphs)
            assert np.array_equal(db.count().per_graph, per_graph_oracle(b))


def test_batch_with_empty_and_tiny_graphs():
    graphs = [mce.from_edges(np.array([], np.int64), np.array([], np.int64), 5),   # no edges
              mce.from_edges(np.array([0]), np.array([1]), 2),                       # one edge
              mce.gen_er(50, 0.2, 4)]
    rp = np.concatenate([g.row_ptr[:g.n + 1] for g in graphs]).astype(np.int32)
    col = np.concatenate([g.col for g in graphs]).astype(np.int32)
    vo = np.cumsum([0] + [g.n + 1 for g in graphs]).astype(np.int64)
    ao = np.cumsum([0] + [g.m for g in graphs]).astype(np.int64)
    hb = mce.HostGraph(rp, col, int(sum(g.n for g in graphs)), int(col.size), 3, vo, ao)
    with mce.Batch(hb) as db:
        r = db.count()
    assert list(r.per_graph) == [0, 1, oracle.count(graphs[2])[0]]



def _count_host(db, b, **kw):
    rp, col, vo, ao = mce.Batch._arrays(b)
    return db.count_host(rp.ctypes.data, col.ctypes.data, vo.ctypes.data, ao.ctypes.data,
                         b.num_graphs, **kw)


@pytest.mark.parametrize("seed", [3, 4])
def test_batch_count_host_in_parts(seed):
    # > 2^20 arcs: copied in parts, each rebased, peeled and oriented on arrival
    b = mce.gen_chung_lu_batch(160, 64, 8192, 2.3, 8, 32, 5, 5, 40, seed)
    assert b.m >= 1 << 20
    with mce.Batch(b) as db:
        ref = db.count()
        small = mce.gen_chung_lu_batch(6, 64, 512, 2.3, 8, 16, 2, 5, 12, 9)  # one part
        for _ in range(2):  # replay of the captured search after a parted upload
            h = _count_host(db, b)
            assert np.array_equal(h.per_graph, ref.per_graph) and h.total == ref.total
            assert np.array_equal(h.hist, ref.hist)
            assert h.stats["tree_nodes"] == ref.stats["tree_nodes"]
            assert h.stats["degeneracy"] == ref.stats["degeneracy"]
        hs = _count_host(db, small)
        assert np.array_equal(hs.per_graph, per_graph_oracle(small))
        for kw in ({"cuda_graph": 0}, {"sched": mce.SCHED_DEGREE}, {"worker_list": mce.WL_OFF}):
            h = _count_host(db, b, **kw)
            assert np.array_equal(h.per_graph, ref.per_graph), kw
        again = db.count()  # the resident batch after the parted upload
    assert np.array_equal(again.per_graph, ref.per_graph)
    want = per_graph_oracle(mce.gen_chung_lu_batch(16, 64, 8192, 2.3, 8, 32, 5, 5, 40, seed))
    assert np.array_equal(ref.per_graph[:16], want)


def test_batch_count_host_uneven_parts():
    # one graph holds most arcs and empty graphs sit at the part edges
    big = mce.gen_er(60000, 0.0006, 5)
    graphs = [mce.from_edges(np.array([], np.int64), np.array([], np.int64), 3), big,
              mce.from_edges(np.array([], np.int64), np.array([], np.int64), 0),
              mce.gen_er(200, 0.05, 6), mce.from_edges(np.array([0]), np.array([1]), 2)]
    rp = np.concatenate([g.row_ptr[:g.n + 1] for g in graphs]).astype(np.int32)
    col = np.concatenate([g.col for g in graphs]).astype(np.int32)
    vo = np.cumsum([0] + [g.n + 1 for g in graphs]).astype(np.int64)
    ao = np.cumsum([0] + [g.m for g in graphs]).astype(np.int64)
    hb = mce.HostGraph(rp, col, int(sum(g.n for g in graphs)), int(col.size), len(graphs), vo, ao)
    assert hb.m >= 1 << 20
    with mce.Batch(hb) as db:
        ref = db.count()
        h = _count_host(db, hb)
    assert np.array_equal(h.per_graph, ref.per_graph) and h.total == ref.total
    assert list(h.per_graph[[0, 2, 4]]) == [0, 0, 1]
    assert h.per_graph[3] == oracle.count(graphs[3])[0]


def test_batch_peel_numbering_matches_single_graphs():
    # The per-graph peel numbers each graph's rounds as a run on that graph
    # alone: the orientation, hence every tree, equals the single-graph
    # runs'.  Graphs up to 16,384 vertices are peeled in shared memory, the
    # 20,000-vertex one in global memory.
    graphs = [mce.gen_er(20000, 0.0008, 3, 5, 6, 20)]
    b = mce.gen_chung_lu_batch(12, 64, 16384, 2.3, 8, 32, 5, 5, 40, 17)
    graphs += [b.graph(i) for i in range(b.num_graphs)]
    rp = np.concatenate([g.row_ptr[:g.n + 1] for g in graphs]).astype(np.int32)
    col = np.concatenate([g.col for g in graphs]).astype(np.int32)
    vo = np.cumsum([0] + [g.n + 1 for g in graphs]).astype(np.int64)
    ao = np.cumsum([0] + [g.m for g in graphs]).astype(np.int64)
    hb = mce.HostGraph(rp, col, int(sum(g.n for g in graphs)), int(col.size), len(graphs), vo, ao)
    single_nodes, single_counts, degen = 0, [], 0
    for g in graphs:
        with mce.Graph.from_host(g) as dg:
            r = dg.count(worker_list=mce.WL_OFF)
        single_nodes += r.stats["tree_nodes"]
        single_counts.append(r.total)
        degen = max(degen, r.stats["degeneracy"])
    with mce.Batch(hb) as db:
        rb = db.count(worker_list=mce.WL_OFF)
    assert list(rb.per_graph) == single_counts
    assert rb.stats["tree_nodes"] == single_nodes
    assert rb.stats["degeneracy"] == degen


def _concat(graphs):
    rp = np.concatenate([g.row_ptr[:g.n + 1] for g in graphs]).astype(np.int32)
    col = np.concatenate([g.col for g in graphs]).astype(np.int32)
    vo = np.cumsum([0] + [g.n + 1 for g in graphs]).astype(np.int64)
    ao = np.cumsum([0] + [g.m for g in graphs]).astype(np.int64)
    return mce.HostGraph(rp, col, int(sum(g.n for g in graphs)), int(col.size), len(graphs), vo, ao)


def _hub(n, seed):
    """Vertex 0 adjacent to all, in a K8 peeled last: a hub root (n - 8
    earlier neighbours, 7 later ones)."""
    base = mce.gen_er(n, 6.0 / n, seed)
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


@pytest.mark.parametrize("kw", [
    {}, {"sched": mce.SCHED_DEGREE}, {"warps_per_root": 2},
    {"bucket_warps_per_root": (1, 2, 4), "bucket_donate_threshold": (10, 16, 6)},
    {"x_pivot": 1}, {"log_roots": True},  # the last one: one search after all parts
], ids=["plain", "degree", "w2", "buckets", "ipx", "logged"])
def test_batch_count_host_part_by_part_search(kw):
    """Parts searched as they land (hub roots in early and late parts, a
    wide-engine R-MAT graph): per-graph counts equal the resident batch's and
    the oracle's, twice in a row, and the resident count after it too.  The
    batch has 64-bit-row roots (planted cliques of up to 40 vertices), so the
    32-bit hubs share the final 64-bit launch."""
    cl = mce.gen_chung_lu_batch(120, 64, 8192, 2.3, 8, 32, 5, 5, 40, 7)
    graphs = [_hub(3000, 1)] + [cl.graph(i) for i in range(cl.num_graphs)] + \
        [_hub(6000, 2), mce.gen_rmat(11, 16, 0.57, 0.19, 0.19, 3)]
    hb = _concat(graphs)
    assert hb.m >= 1 << 20
    want = np.array([oracle.count(g)[0] for g in graphs], np.uint64)
    with mce.Batch(hb) as db:
        ref = db.count(**{k: v for k, v in kw.items() if k != "log_roots"})
        assert np.array_equal(ref.per_graph, want)
        assert ref.stats["class_roots"][1] > 0  # 33 <= d+ <= 64
        for _ in range(2):
            h = _count_host(db, hb, **kw)
            assert h.stats["error_flags"] == 0
            assert np.array_equal(h.per_graph, want) and h.total == int(want.sum())
            assert np.array_equal(h.hist, ref.hist)
        again = db.count()
    assert np.array_equal(again.per_graph, want)
