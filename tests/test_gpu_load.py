"""Device .bel loader (mce_bel_load) against the host reader + upload."""
import numpy as np
import pytest

import mce_b200 as mce
import oracle

pytestmark = pytest.mark.gpu


def same_graph(path):
    h = mce.bel_read(path)
    with mce.Graph.load_bel(path) as d, mce.Graph.from_host(h) as u:
        assert (d.n, d.m) == (h.n, h.m)
        # identical CSR <=> identical split CSR (same peel, same orientation)
        sd, cd = d.split_csr()
        su, cu = u.split_csr()
        assert np.array_equal(sd, su) and np.array_equal(cd, cu)
        rd, ru = d.count(), u.count()
    assert rd.total == ru.total and np.array_equal(rd.hist, ru.hist)
    return h, rd.total


@pytest.mark.parametrize("maker", [
    lambda: mce.gen_er(3000, 0.01, 3, 10, 6, 20),
    lambda: mce.gen_rmat(11, 16, 0.57, 0.19, 0.19, 7),
    lambda: mce.gen_ba(300000, 8, 9),            # 4.8e6 records: three staging chunks
])
def test_load_matches_host_reader(tmp_path, maker):
    g = maker()
    path = str(tmp_path / "g.bel")
    mce.bel_write(path, g)
    h, total = same_graph(path)
    if h.n <= 5000:
        assert total == oracle.count(h)[0]


def test_load_leading_isolated_vertices(tmp_path):
    # edges only among vertices 5..8: rows 0..4 are empty
    src = np.array([5, 6, 6, 7, 7, 8], np.int64)
    dst = np.array([6, 5, 7, 6, 8, 7], np.int64)
    g = mce.from_edges(src, dst, 9)
    path = str(tmp_path / "g.bel")
    mce.bel_write(path, g)
    h, total = same_graph(path)
    assert h.n == 9 and total == 3


def test_load_rejects_bad_files(tmp_path):
    p = tmp_path / "bad.bel"

    def code(recs=None, raw=None):
        p.write_bytes(raw if raw is not None else np.array(recs, np.uint64).tobytes())
        with pytest.raises(mce.MceError) as e:
            mce.Graph.load_bel(str(p))
        return e.value.code

    assert code(raw=b"\0" * 25) == mce.EFORMAT                       # not whole records
    assert code([[1, 2, 0], [2, 1, 0]]) == mce.EFORMAT               # sources out of order
    assert code([[1, 0, 0], [0, 1, 0], [1, 1, 0]]) == mce.EFORMAT    # self-loop (1, 1)
    assert code([[1, 0, 0], [1, 0, 0], [0, 1, 0]]) == mce.EFORMAT    # duplicate record
    assert code([[5, 0, 0], [0, 1, 0]]) == mce.EFORMAT               # destination >= n
    assert code([[1, 0, 0], [0, 1 << 40, 0]]) == mce.EFORMAT         # id above 2^31
    with pytest.raises(mce.MceError) as e:
        mce.Graph.load_bel(str(tmp_path / "missing.bel"))
    assert e.value.code == mce.EIO


# ---------------------------------------------------------------------------
# text edge lists: the device converter against the host converter
# ---------------------------------------------------------------------------
EDGE_CASES = (
    b"# comment line\n% another\n1 2\n2 3\r\n3\t4\n  5 6\n7 7\n8 +9\n10 -1\n"
    b"11 99999999999999999999999\n12 4294967308\n13 x\n14 -x\n15\n\n16 17 trailing\n"
    b"0 1\n1 2\n2 1\n18\x0019\n20 21\n"
    + b"22" + b" " * 70000 + b"23\n"          # second number past the 65,535-byte window
    + b"24 25" + b"x" * 70000 + b"\n"         # edge, then a long tail
    + b"#" + b"y" * 70000 + b"\n26 27\n"      # long comment, then an edge
    + b"28 29"                                # last line without a newline
)


def text_of(src, dst, comments=0, seed=0):
    rng = np.random.default_rng(seed)
    lines = [f"{a} {b}" for a, b in zip(src.tolist(), dst.tolist())]
    for i in rng.integers(0, len(lines) + 1, comments):
        lines.insert(int(i), "# c")
    return ("\n".join(lines) + "\n").encode()


def both_converters(tmp_path, data):
    txt = tmp_path / "g.txt"
    txt.write_bytes(data)
    hb, db = tmp_path / "h.bel", tmp_path / "d.bel"
    hn = mce.convert_to_bel(str(txt), str(hb))
    dn = mce.convert_to_bel(str(txt), str(db), device=0)
    assert hn == dn
    assert hb.read_bytes() == db.read_bytes()
    return str(txt), str(hb), hn


def test_convert_device_edge_cases(tmp_path):
    _, bel, (n, e) = both_converters(tmp_path, EDGE_CASES)
    rec = np.fromfile(bel, np.uint64).reshape(-1, 3)
    pairs = {(int(s), int(d)) for d, s, _ in rec}
    assert n == 0  # the max id is 2^64-1, so max id + 1 wraps to 0
    for a, b in [(1, 2), (2, 3), (3, 4), (8, 9), (16, 17), (0, 1), (20, 21), (24, 25),
                 (26, 27), (28, 29), (12, 12)]:
        assert (a, b) in pairs and (b, a) in pairs
    for a, b in [(5, 6), (7, 7), (13, 14), (18, 19), (22, 23)]:
        assert (a, b) not in pairs
    assert (10, 2**32 - 1) in pairs and (11, 2**32 - 1) in pairs  # -1 and overflow narrow alike
    assert e == len(rec) // 2


def test_convert_device_empty_and_comments_only(tmp_path):
    assert both_converters(tmp_path, b"")[2] == (1, 0)
    assert both_converters(tmp_path, b"# nothing\n\n%\n")[2] == (1, 0)


@pytest.mark.parametrize("maker,comments", [
    (lambda: mce.gen_er(3000, 0.01, 3, 10, 6, 20), 50),
    (lambda: mce.gen_rmat(12, 16, 0.57, 0.19, 0.19, 7), 0),
])
def test_text_load_matches_bel_path(tmp_path, maker, comments):
    g = maker()
    src = np.repeat(np.arange(g.n), np.diff(g.row_ptr[:g.n + 1]))
    dst = g.col[:g.m]
    keep = src < dst                     # each undirected edge once, as SNAP lists them
    rng = np.random.default_rng(1)
    perm = rng.permutation(int(keep.sum()))
    data = text_of(src[keep][perm], dst[keep][perm], comments)
    txt, bel, (n, e) = both_converters(tmp_path, data)
    assert e == g.m // 2
    with mce.Graph.load_text(txt) as t, mce.Graph.load_bel(bel) as b:
        # trailing isolated vertices vanish in both (n = max id + 1)
        top = int(max(src[keep].max(), dst[keep].max()))
        assert (t.n, t.m) == (b.n, b.m) == (top + 1, g.m)
        st, ct = t.split_csr()
        sb, cb = b.split_csr()
        assert np.array_equal(st, sb) and np.array_equal(ct, cb)
        rt, rb = t.count(), b.count()
    assert rt.total == rb.total and np.array_equal(rt.hist, rb.hist)
    if g.n <= 5000:
        assert rt.total == oracle.count(g)[0]


def test_convert_device_many_chunks(tmp_path):
    # > 64 MiB of text (two staging buffers reused) and > 2^21 records out
    rng = np.random.default_rng(5)
    src = rng.integers(0, 3_000_000, 5_200_000)
    dst = rng.integers(0, 3_000_000, 5_200_000)
    data = text_of(src, dst)
    assert len(data) > (64 << 20) + 1
    _, _, (n, e) = both_converters(tmp_path, data)
    assert n == int(max(src.max(), dst.max())) + 1 and e > 5_000_000


def test_text_load_rejects(tmp_path):
    p = tmp_path / "t.txt"

    def code(data):
        p.write_bytes(data)
        with pytest.raises(mce.MceError) as e:
            mce.Graph.load_text(str(p))
        return e.value.code

    assert code(b"1 2\n5 4294967301\n") == mce.EFORMAT     # 5 and 2^32+5 narrow to one vertex
    assert code(b"1 2\n3 2147483650\n") == mce.ELIMIT      # id above the int32 CSR
    with pytest.raises(mce.MceError) as e:
        mce.Graph.load_text(str(tmp_path / "missing.txt"))
    assert e.value.code == mce.EIO
    p.write_bytes(b"# no edges\n")
    with mce.Graph.load_text(str(p)) as g:
        assert (g.n, g.m) == (0, 0) and g.count().total == 0
