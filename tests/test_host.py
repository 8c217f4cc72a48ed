"""Host-side library code: generators, .bel I/O, CSR checks, exported symbols, CLI."""
import ctypes
import glob
import os
import re
import subprocess

import numpy as np
import pytest

import mce_b200 as mce
import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "mce-gpu_b200", "bin", "parallel_mce_on_gpus")


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^[A-Za-z_][\w \*]*?\b(mce_\w+)\s*\(", src, flags=re.M):
            names.add(m.group(1))
    return sorted(names)


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(mce.LIB_PATH)
    names = declared_functions()
    assert len(names) > 20
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_generators_deterministic():
    a = mce.gen_rmat(12, 16, 0.57, 0.19, 0.19, 7)
    b = mce.gen_rmat(12, 16, 0.57, 0.19, 0.19, 7)
    c = mce.gen_rmat(12, 16, 0.57, 0.19, 0.19, 8)
    assert np.array_equal(a.col, b.col) and np.array_equal(a.row_ptr, b.row_ptr)
    assert not (a.m == c.m and np.array_equal(a.col, c.col))
    for g in (a, mce.gen_er(2000, 0.01, 1, 5), mce.gen_ba(5000, 4, 3, 5, 5, 10)):
        assert mce.validate(g) == 0


def test_er_config_shape():
    """ER(10000, 0.002) + 20 planted cliques of size 6..12 (the small plain config)."""
    g = mce.gen_er(10000, 0.002, 1, 20, 6, 12)
    assert g.n == 10000
    assert 190_000 < g.m < 215_000  # ~1e5 edges from G(n,p) + planted pairs


def test_chung_lu_batch_layout():
    b = mce.gen_chung_lu_batch(16, 64, 2048, 2.3, 8, 32, 5, 5, 40, 11)
    assert b.num_graphs == 16
    assert b.vtx_offsets[-1] == b.n + 16 and b.arc_offsets[-1] == b.m
    u = mce.union(b)
    assert mce.validate(u) == 0
    tot_u = oracle.count(u)[0]
    assert tot_u == sum(oracle.count(b.graph(i))[0] for i in range(16))


def test_permutation_invariance_oracle():
    g = mce.gen_er(800, 0.03, 2, 6, 6, 14)
    p = mce.permute(g, 99)
    assert mce.validate(p) == 0
    t, h, _ = oracle.count(g)
    tp, hp, _ = oracle.count(p)
    assert t == tp and np.array_equal(h, hp)


def test_bel_roundtrip(tmp_path):
    g = mce.gen_er(500, 0.05, 3, 3, 5, 9)
    path = str(tmp_path / "g.bel")
    mce.bel_write(path, g)
    assert os.path.getsize(path) == 24 * g.m
    raw = np.fromfile(path, dtype=np.uint64).reshape(-1, 3)
    # record layout: dst, src, 0 ; sorted by (src, dst)
    assert np.all(raw[:, 2] == 0)
    src, dst = raw[:, 1], raw[:, 0]
    assert np.all(np.diff(src.astype(np.int64)) >= 0)
    h = mce.bel_read(path)
    # n = max src + 1 (trailing isolated vertices vanish, as in the reference)
    nmax = int(src.max()) + 1
    assert h.n == nmax and h.m == g.m
    assert np.array_equal(h.col, g.col)
    assert np.array_equal(h.row_ptr[:nmax + 1], g.row_ptr[:nmax + 1])


def test_bel_rejects_bad_files(tmp_path):
    p = tmp_path / "bad.bel"
    p.write_bytes(b"\0" * 25)
    with pytest.raises(mce.MceError) as e:
        mce.bel_read(str(p))
    assert e.value.code == mce.EFORMAT
    # unsorted sources
    recs = np.array([[1, 2, 0], [2, 1, 0]], np.uint64)  # (dst, src): src 2 then 1
    p.write_bytes(recs.tobytes())
    with pytest.raises(mce.MceError):
        mce.bel_read(str(p))
    with pytest.raises(mce.MceError) as e:
        mce.bel_read(str(tmp_path / "missing.bel"))
    assert e.value.code == mce.EIO


def test_convert_to_bel(tmp_path):
    txt = tmp_path / "g.txt"
    txt.write_text("# comment\n0 1\n1 2\n2 0\n2 2\n3 1\n% other\n1 0\n")
    bel = str(tmp_path / "g.bel")
    n, e = mce.convert_to_bel(str(txt), bel)
    assert (n, e) == (4, 4)  # edges {01, 12, 02, 13}; self-loop dropped; duplicate merged
    g = mce.bel_read(bel)
    assert g.n == 4 and g.m == 8
    assert list(g.col) == [1, 2, 0, 2, 3, 0, 1, 1]
    assert oracle.count(g)[0] == 2  # triangle 012 + edge 13


def _scan_llu(line, p):
    """One strtoull-style %llu conversion at line[p:] (bytes): leading blanks,
    optional sign, decimal digits, ULLONG_MAX on overflow, '-' negating
    modulo 2^64.  Returns (value, next position) or None."""
    while p < len(line) and line[p] in b" \t\v\f\r\n":
        p += 1
    neg = False
    if p < len(line) and line[p] in b"+-":
        neg = line[p] == ord("-")
        p += 1
    q = p
    while q < len(line) and 48 <= line[q] <= 57:
        q += 1
    if q == p:
        return None
    x = int(line[p:q])
    x = 2**64 - 1 if x >= 2**64 else ((-x) % 2**64 if neg else x)
    return x, q


def _convert_model(data):
    """graph::convert_to_bel's result (include/fileop.h:13-79) for a text
    file: (n, undirected edges, sorted unique (src, dst) arcs), reading at
    most the first 65,535 bytes of each line; a NUL byte ends a line's text."""
    arcs, mx, any_edge = set(), 0, False
    for raw in data.split(b"\n"):
        line = raw[:65535].split(b"\0")[0]
        if not line or not (48 <= line[0] <= 57):
            continue
        a = _scan_llu(line, 0)
        b = _scan_llu(line, a[1]) if a else None
        if not (a and b) or a[0] == b[0]:
            continue
        s, d = a[0], b[0]
        arcs.add((s & 0xFFFFFFFF, d & 0xFFFFFFFF))
        arcs.add((d & 0xFFFFFFFF, s & 0xFFFFFFFF))
        mx, any_edge = max(mx, s, d), True
    n = ((mx + 1) % 2**64) if any_edge else 1
    return n if n < 2**63 else n - 2**64, len(arcs) // 2, sorted(arcs)


def test_convert_to_bel_line_semantics(tmp_path):
    data = (b"# comment\n% other\n1 2\n2 3\r\n3\t4\n  5 6\n7 7\n8 +9\n10 -1\n"
            b"11 99999999999999999999999\n12 4294967308\n13 x\n14 -x\n15\n\n16 17 tail\n"
            b"0 1\n1 2\n2 1\n18\x0019\n20 21\n"
            + b"22" + b" " * 70000 + b"23\n"
            + b"24 25" + b"x" * 70000 + b"\n"
            + b"#" + b"y" * 70000 + b"\n26 27\n"
            + b"28 29")
    txt = tmp_path / "g.txt"
    txt.write_bytes(data)
    bel = tmp_path / "g.bel"
    n, e = mce.convert_to_bel(str(txt), str(bel))
    want_n, want_e, want_arcs = _convert_model(data)
    assert (n, e) == (want_n, want_e)
    rec = np.fromfile(str(bel), np.uint64).reshape(-1, 3)
    assert [(int(s), int(d)) for d, s, _ in rec] == want_arcs
    assert all(int(z) == 0 for _, _, z in rec)


def test_validate_rejects_asymmetric():
    rp = np.array([0, 1, 1], np.int32)
    col = np.array([1], np.int32)
    g = mce.HostGraph(rp, col, 2, 1)
    assert mce.validate(g) == mce.EFORMAT


def ego_reference(g, seed, cap):
    """The ego-graph definition in plain Python: seed, neighbours in row
    order, then 2-hop vertices in discovery order, at most cap; ascending
    relabel.  Returns (sorted vertex ids, set of edges in original ids)."""
    rp, col = g.row_ptr, g.col
    verts, seen = [seed], {seed}
    for w in col[rp[seed]:rp[seed + 1]]:
        if len(verts) >= cap:
            break
        if int(w) not in seen:
            seen.add(int(w))
            verts.append(int(w))
    k1 = len(verts)
    for u in verts[1:k1]:
        for w in col[rp[u]:rp[u + 1]]:
            if len(verts) >= cap:
                break
            if int(w) not in seen:
                seen.add(int(w))
                verts.append(int(w))
    vs = sorted(verts)
    edges = {(int(a), int(b)) for a in vs for b in col[rp[a]:rp[a + 1]] if int(b) in seen and a < b}
    return vs, edges


@pytest.mark.parametrize("seed,cap", [(7, 64), (0, 2), (3, 400), (11, 150)])
def test_ego_subgraph(seed, cap):
    g = mce.gen_ba(400, 4, 5, planted=3, cmin=6, cmax=10)
    eg, vmap = mce.ego_subgraph(g, seed, cap)
    assert mce.validate(eg) == 0
    vs, edges = ego_reference(g, seed, cap)
    assert list(vmap) == vs and seed in vs
    got = {(int(vmap[u]), int(vmap[w])) for u in range(eg.n)
           for w in eg.col[eg.row_ptr[u]:eg.row_ptr[u + 1]] if u < w}
    assert got == edges


@pytest.mark.skipif(not os.path.exists(CLI), reason="CLI not built")
class TestCli:
    def run(self, *args):
        return subprocess.run([CLI, *args], capture_output=True, text=True, timeout=60)

    def test_missing_task(self):
        r = self.run("-g", "x.bel")
        assert r.returncode == 0 and "Must specify -m option" in r.stderr

    def test_bad_options_exit_zero(self):
        for args, msg in [(("-m", "foo"), "Unrecognized -m option"),
                          (("-m", "mce", "-g", "a", "-d", "0", "-p", "l3"), "Unrecognized -p option"),
                          (("-m", "mce", "-g", "a", "-d", "0", "-p", "l1", "-i", "q"), "Unrecognized -i option"),
                          (("-m", "mce", "-g", "a", "-p", "l1", "-i", "p", "-w", "wl"), "Must specify -d option"),
                          (("-m", "mce-bd-eval", "-g", "a", "-d", "0", "-p", "l1", "-i", "p", "-w", "nowl"),
                           "No breakdown for kernels without worker list")]:
            r = self.run(*args)
            assert r.returncode == 0 and msg in r.stderr, (args, r.stderr)

    def test_help(self):
        r = self.run("-h")
        assert r.returncode == 0 and "Usage:" in r.stderr

    def test_convert_task(self, tmp_path):
        txt = tmp_path / "g.txt"
        txt.write_text("0 1\n1 2\n2 0\n")
        bel = tmp_path / "g.bel"
        r = self.run("-m", "convert", "-g", str(txt), "-r", str(bel))
        assert r.returncode == 0
        assert "Main Task = convert" in r.stdout and "n = 3 and m = 3" in r.stdout
        assert os.path.getsize(bel) == 6 * 24


def test_tune_table_lookup(tmp_path):
    t = tmp_path / "tune.txt"
    assert mce.tune_lookup(str(t), "n10-a3-k4") is None  # no table yet
    t.write_text("# mce autotune table v1\n"
                 "n10-a3-k4 1 1024 6 64 -1 1.5 2.0\n"
                 "b12-n23-a4-k7 2 64 16 32 64 100.0 110.0\n")
    assert mce.tune_lookup(str(t), "n10-a3-k4") == dict(
        worker_list=1, donate_after=1024, donate_threshold=6, bitmap_width=64, peel_solo_max=-1,
        wide_blocks=4, x_pivot=0, warps_per_root=0, bucket_warps_per_root=(0, 0, 0),
        bucket_donate_threshold=(0, 0, 0), bucket_donate_after=(0, 0, 0))
    # (a v1 line: no wide_blocks or x_pivot column, no buckets)
    assert mce.tune_lookup(str(t), "b12-n23-a4-k7")["peel_solo_max"] == 64
    assert mce.tune_lookup(str(t), "n11-a3-k4") is None
    t.write_text("# mce autotune table v2\nn14-a4-k6 2 1024 10 32 -1 8 900.0 1100.0\n")
    assert mce.tune_lookup(str(t), "n14-a4-k6")["wide_blocks"] == 8
    t.write_text("# mce autotune table v3\nn14-a4-k6 2 1024 10 32 -1 8 1 800.0 1100.0\n")
    assert mce.tune_lookup(str(t), "n14-a4-k6")["x_pivot"] == 1
    # v4: a line per bucket of roots (engine class), before or after the class line
    t.write_text("# mce autotune table v4\n"
                 "b12-n23-a4-k5:b64 2 6 1024 3.1 4.0\n"
                 "b12-n23-a4-k5 2 256 10 32 -1 4 0 45.0 47.4\n"
                 "b12-n23-a4-k5:b32 1 10 256 30.0 30.0\n"
                 "n9-a3-k4:wide 4 16 64 1.0 2.0\n")  # buckets without a class line: none
    r = mce.tune_lookup(str(t), "b12-n23-a4-k5")
    assert r["bucket_warps_per_root"] == (1, 2, 0)
    assert r["bucket_donate_threshold"] == (10, 6, 0)
    assert r["bucket_donate_after"] == (256, 1024, 0)
    assert r["donate_after"] == 256
    assert mce.tune_lookup(str(t), "n9-a3-k4") is None


def test_device_file_paths_fail_loudly_without_a_device(tmp_path):
    # no silent host fallback: the device converter and loader report MCE_ENODEV
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is visible")
    txt = tmp_path / "g.txt"
    txt.write_text("0 1\n1 2\n")
    with pytest.raises(mce.MceError) as e:
        mce.convert_to_bel(str(txt), str(tmp_path / "g.bel"), device=0)
    assert e.value.code == mce.ENODEV
    with pytest.raises(mce.MceError) as e:
        mce.Graph.load_text(str(txt))
    assert e.value.code == mce.ENODEV
