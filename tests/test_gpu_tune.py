"""Autotuner: tuned settings never change the count; the table round-trips."""
import numpy as np
import pytest

import mce_b200 as mce
import oracle

pytestmark = pytest.mark.gpu


def test_autotune_graph(tmp_path):
    table = str(tmp_path / "tune.txt")
    hg = mce.gen_rmat(11, 16, 0.57, 0.19, 0.19, 7)
    want = oracle.count(hg)[0]
    with mce.Graph.from_host(hg) as g:
        r = g.autotune(table, reps=1)
        assert r["key"] == g.shape_key() and not r["from_table"] and r["trials_run"] >= 5
        assert g.count(**r["best"]).total == want
        again = g.autotune(table, reps=1)
    assert again["from_table"] and again["best"] == r["best"] and again["trials_run"] == 0
    assert mce.tune_lookup(table, r["key"]) == r["best"]


def test_autotune_batch(tmp_path):
    table = str(tmp_path / "tune.txt")
    b = mce.gen_chung_lu_batch(24, 64, 2048, 2.3, 8, 32, 5, 5, 40, 3)
    want = np.array([oracle.count(b.graph(i))[0] for i in range(b.num_graphs)], np.uint64)
    with mce.Batch(b) as db:
        r = db.autotune(table, reps=1)
        assert r["key"].startswith("b4-")
        res = db.count(**r["best"])
    assert np.array_equal(res.per_graph, want)
    assert mce.tune_lookup(table, r["key"]) == r["best"]
    # a line per bucket of roots that the batch has (its narrow roots at least)
    lines = open(table).read().splitlines()
    assert any(l.startswith(r["key"] + ":b32 ") for l in lines)
    assert r["best"]["bucket_warps_per_root"][0] in (1, 2, 4)
