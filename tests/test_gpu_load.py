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
