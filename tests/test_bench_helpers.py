"""bench.py's host-side figures: the algorithmic bytes of each stage against
a plain loop over the oriented CSR, and the rule that a committed ncu figure
is used only while the kernel sources it was captured on are unchanged."""
import json
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import bench  # noqa: E402
import oracle  # noqa: E402

import mce_b200 as mce  # noqa: E402


def test_algorithmic_bytes_match_a_loop():
    g = mce.gen_er(300, 0.04, 5)
    split, cs = oracle.prepare(g)
    rp = g.row_ptr[:g.n + 1].astype(np.int64)
    dplus = [int(rp[v + 1] - split[v]) for v in range(g.n)]
    stage_b = 0
    with_rows = 0
    for r in range(g.n):
        later = cs[split[r]:rp[r + 1]]
        stage_b += 4 * (len(later) + sum(dplus[v] for v in later)) + 8 * len(later)
        if dplus[r] > 0:
            nbrs = g.col[rp[r]:rp[r + 1]]
            with_rows += 8 + 4 * len(nbrs) + sum(8 + 4 * dplus[v] for v in nbrs)
    ab = bench.algorithmic_bytes(g, np.asarray(split), np.asarray(cs))
    assert ab["stage_a"] == 24 * g.m + 12 * (g.n + 1)
    assert ab["stage_b"] == stage_b
    assert ab["search_with_earlier_rows"] == with_rows


def test_profile_figures_drop_stale_captures(monkeypatch, tmp_path):
    csrc = tmp_path / "mce-gpu_b200" / "csrc"
    csrc.mkdir(parents=True)
    (csrc / "a.cu").write_text("kernel A\n")
    (csrc / "b.cu").write_text("kernel B\n")
    monkeypatch.setattr(bench, "ROOT", str(tmp_path))
    h_a = bench.kernel_source_hash(["a.cu"])
    (tmp_path / "profiles").mkdir()
    (tmp_path / "profiles" / "traffic.json").write_text(json.dumps({
        "batch:fresh": {"value": 7, "hash": h_a, "sources": ["a.cu"]},
        "batch:stale": {"value": 9, "hash": "0" * 16, "sources": ["b.cu"]},
        "ba:other": {"value": 1, "hash": h_a, "sources": ["a.cu"]},
    }))
    out, note = bench.profile_figures("batch")
    assert out == {"fresh": 7} and "stale" in note
    (csrc / "a.cu").write_text("kernel A, changed\n")  # the capture no longer applies
    out, note = bench.profile_figures("batch")
    assert out == {} and "fresh" in note and "stale" in note
    assert bench.profile_figures("rmat") == ({}, None)
