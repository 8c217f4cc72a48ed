"""Parity against the reference binary's own output (tests/golden/reference_counts.json).

The fixture holds, for seeded graphs, the count and degeneracy printed by the
reference (built from its sources, run on a B200 by
tests/golden/make_ref_golden.py).  The CPU test pins the oracle to it; the
GPU test pins the CUDA path to it.
"""
import json
import os

import pytest

import mce_b200 as mce
import oracle

HERE = os.path.dirname(os.path.abspath(__file__))
with open(os.path.join(HERE, "golden", "reference_counts.json")) as f:
    GOLD = json.load(f)["graphs"]


def make(entry):
    kw = entry["args"]
    if entry["generator"] == "chung_lu_union":
        return mce.union(mce.gen_chung_lu_batch(*kw.values()))
    return getattr(mce, entry["generator"])(*kw.values())


@pytest.mark.parametrize("name", sorted(GOLD))
def test_oracle_matches_reference(name):
    e = GOLD[name]
    g = make(e)
    assert (g.n, g.m) == (e["n"], e["arcs"])
    total, _, degen = oracle.count(g)
    assert total == e["reference_count"]
    assert degen == e["reference_max_core"]


@pytest.mark.gpu
@pytest.mark.parametrize("name", sorted(GOLD))
def test_gpu_matches_reference(name):
    e = GOLD[name]
    g = make(e)
    with mce.Graph.from_host(g) as dg:
        r = dg.count()
    assert r.total == e["reference_count"]
    assert r.stats["degeneracy"] == e["reference_max_core"]
