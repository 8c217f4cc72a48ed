"""Serving sessions (mce_serve_*): every answer against the oracle's count
of the host-built ego graph, alone and mixed with other requests."""
import time

import numpy as np
import pytest

import mce_b200 as mce
import oracle

pytestmark = pytest.mark.gpu


def ego_count(hg, seed, cap):
    eg, _ = mce.ego_subgraph(hg, int(seed), cap)
    return oracle.count(eg)[0], eg.n, eg.m


@pytest.fixture(scope="module")
def ba():
    hg = mce.gen_ba(20000, 6, 31, planted=30, cmin=8, cmax=40)
    g = mce.Graph.from_host(hg)
    yield hg, g
    g.close()


@pytest.mark.parametrize("cap", [64, 1024, 4096])
def test_serve_counts_match_oracle(ba, cap):
    hg, g = ba
    rng = np.random.default_rng(cap)
    hubs = np.argsort(np.diff(hg.row_ptr[:hg.n + 1]))[-4:]  # the widest 2-hop neighbourhoods
    seeds = np.concatenate([rng.integers(0, hg.n, 60), hubs]).astype(np.int64)
    with mce.Serve(g, ego_cap=cap) as s:
        res, lat = s.run(seeds, timeout_ms=120000)
        st = s.stats()
    # one launch per slot class (two when the cap turns the 256-thread class on)
    assert st["served"] == len(seeds) and st["kernel_launches"] == (2 if st["small_slots"] else 1)
    assert (st["small_slots"] > 0) == (cap > 2048)
    for r, seed in zip(res, seeds):
        want, n, m = ego_count(hg, seed, cap)
        assert r["status"] == mce.OK and r["seed"] == seed
        assert (int(r["count"]), int(r["ego_n"]), int(r["ego_arcs"])) == (want, n, m), seed
    assert np.all(lat > 0)


def test_serve_alone_equals_mixed():
    hg = mce.gen_rmat(12, 16, 0.57, 0.19, 0.19, 7)
    seeds = np.random.default_rng(3).integers(0, hg.n, 48).astype(np.int64)
    with mce.Graph.from_host(hg) as g:
        with mce.Serve(g, ego_cap=512, slots=3) as s:
            alone = [s.wait(s.submit(int(x)))["count"] for x in seeds]
            mixed, _ = s.run(seeds, timeout_ms=120000)  # all admitted at once
            spaced, _ = s.run(seeds, np.arange(len(seeds)) * 50.0, 120000)  # open-loop arrivals
    assert [int(c) for c in mixed["count"]] == alone
    assert [int(c) for c in spaced["count"]] == alone
    for seed, c in zip(seeds[:12], alone):
        assert c == ego_count(hg, seed, 512)[0]


def test_serve_bad_seed_and_limits():
    # a 300-clique: its first-peeled vertex has 299 later neighbours
    hg = mce.gen_er(2000, 0.002, 5, planted=1, cmin=300, cmax=300)
    deg = np.diff(hg.row_ptr[:hg.n + 1])
    member = int(np.argmax(deg))
    # a vertex whose ego graph stays clear of the clique
    small = next(v for v in range(hg.n)
                 if deg[v] > 0 and deg[mce.ego_subgraph(hg, v, 1024)[1]].max() < 100)
    with mce.Graph.from_host(hg) as g:
        with mce.Serve(g, ego_cap=1024, max_arcs=1 << 20) as s:
            r_bad = s.wait(s.submit(-1))
            r_big = s.wait(s.submit(hg.n))
            r_wide = s.wait(s.submit(member))
            r_ok = s.wait(s.submit(small))  # the session keeps serving after failures
        with mce.Serve(g, ego_cap=1024, max_arcs=1000) as s:
            r_arcs = s.wait(s.submit(member))
    assert r_bad["status"] == mce.EINVAL and r_big["status"] == mce.EINVAL
    assert r_wide["status"] == mce.ELIMIT and r_wide["limits"] & mce.SERVE_TOO_WIDE
    assert r_arcs["status"] == mce.ELIMIT and r_arcs["limits"] == mce.SERVE_OVER_ARCS
    assert r_ok["status"] == mce.OK and r_ok["count"] == ego_count(hg, small, 1024)[0]
    assert r_ok["limits"] == 0


def test_serve_node_budget():
    hg = mce.gen_er(400, 0.25, 8)  # every ego graph is the whole dense graph
    want = ego_count(hg, 3, 1024)[0]
    with mce.Graph.from_host(hg) as g:
        with mce.Serve(g, ego_cap=1024, max_nodes=500) as s:
            cut = s.wait(s.submit(3))
        with mce.Serve(g, ego_cap=1024) as s:
            full = s.wait(s.submit(3))
    assert cut["status"] == mce.ELIMIT and cut["limits"] == mce.SERVE_OVER_BUDGET
    assert full["status"] == mce.OK and full["count"] == want and want > 5000


def test_serve_ring_full_and_idle_relaunch():
    hg = mce.gen_ba(5000, 4, 9)
    with mce.Graph.from_host(hg) as g:
        with mce.Serve(g, ego_cap=128, ring=4, idle_ms=50) as s:
            ids = [s.submit(i) for i in range(4)]
            with pytest.raises(mce.MceError) as e:
                s.submit(4)
            assert e.value.code == mce.ELIMIT
            first = s.wait(ids[0])
            ids.append(s.submit(4))  # a taken answer frees its entry
            rest = [s.wait(i) for i in ids[1:]]
            time.sleep(0.5)          # every slot leaves after 50 ms idle
            assert s.stats()["running"] == 0
            again = s.wait(s.submit(0))
            st = s.stats()
    assert st["kernel_launches"] == 2 and st["served"] == 6
    assert again["count"] == first["count"] == ego_count(hg, 0, 128)[0]
    for i, r in enumerate(rest, start=1):
        assert r["count"] == ego_count(hg, i, 128)[0]


def test_serve_poll_contract():
    hg = mce.gen_ba(3000, 4, 2)
    with mce.Graph.from_host(hg) as g:
        with mce.Serve(g, ego_cap=256) as s:
            rid = s.submit(5)
            r = None
            t0 = time.time()
            while r is None and time.time() - t0 < 30:
                r = s.poll(rid)
            assert r is not None and r["count"] == ego_count(hg, 5, 256)[0]
            with pytest.raises(mce.MceError):
                s.poll(rid)  # an answer is taken once
            pending = [s.submit(i) for i in range(20)]
        # closing with unpolled requests finishes them and frees the session
        assert len(pending) == 20


def test_serve_idle_slots_help_large_requests(ba):
    hg, g = ba
    deg = np.diff(hg.row_ptr[:hg.n + 1])
    seeds = [int(x) for x in np.argsort(deg)[-8:]]  # hubs: ego graphs at the cap
    with mce.Serve(g, ego_cap=4096) as s:
        got = [s.wait(s.submit(x)) for x in seeds]  # one at a time: the other slots idle
        st = s.stats()
    for r, x in zip(got, seeds):
        want, n, m = ego_count(hg, x, 4096)
        assert r["status"] == mce.OK and n >= 1024
        assert (int(r["count"]), int(r["ego_n"])) == (want, n)
    assert st["helps"] > 0


def test_serve_footprint_classes(ba):
    """Requests whose footprint bound fits small_cap go to the 256-thread
    slots (id bit 0 set) once every whole-block slot holds a request, the
    others to the whole-block slots; every answer matches the oracle either
    way."""
    hg, g = ba
    deg = np.diff(hg.row_ptr[:hg.n + 1]).astype(np.int64)
    bound = deg + np.array([deg[hg.col[hg.row_ptr[v]:hg.row_ptr[v + 1]]].sum()
                            for v in range(hg.n)])
    small = np.flatnonzero(bound + 1 <= 256)[:40]
    large = np.argsort(deg)[-6:]
    seeds = np.concatenate([small, large, small[:10]]).astype(np.int64)
    with mce.Serve(g, ego_cap=2048, small_cap=256, big_slots=4) as s:
        ids = [s.submit(int(x)) for x in seeds]
        got = [s.wait(i) for i in ids]
        res, _ = s.run(seeds, timeout_ms=120000)
        st = s.stats()
    assert st["small_cap"] == 256 and st["small_slots"] > 0
    assert st["slots"] == 4 + st["small_slots"]
    assert 1 <= st["peak_in_flight"] <= len(seeds)
    cls = [rid & 1 for rid in ids]
    fits = [bool(bound[x] + 1 <= 256) for x in seeds]
    assert cls[:4] == [0] * 4  # the four whole-block slots take the first ones
    assert cls[4:] == [1 if f else 0 for f in fits[4:]]
    for r, rr, x in zip(got, res, seeds):
        want, n, m = ego_count(hg, x, 2048)
        assert r["status"] == mce.OK and (int(r["count"]), int(r["ego_n"])) == (want, n), x
        assert int(rr["count"]) == want
