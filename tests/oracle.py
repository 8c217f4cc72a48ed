"""ctypes wrapper of oracle/liboracle.so - the CPU checker (tests only)."""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "oracle", "liboracle.so")
if not os.path.exists(LIB):
    subprocess.run(["make", "-C", os.path.join(ROOT, "oracle")], check=True,
                   stdout=subprocess.DEVNULL)
_o = C.CDLL(LIB)
_P = C.c_void_p
_o.oracle_peel.argtypes = [C.c_int64, _P, _P, _P, _P, _P]
_o.oracle_orient.argtypes = [C.c_int64, _P, _P, _P, _P, _P]
_o.oracle_mce.argtypes = [C.c_int64, _P, _P, _P, C.c_int64, C.c_int64, C.c_int64, C.c_int,
                          _P, _P, C.c_int, _P, _P]
_o.oracle_mce_ops.argtypes = [C.c_int64, _P, _P, _P, C.c_int64, C.c_int64, C.c_int64, C.c_int,
                              _P, _P, C.c_int, _P, _P, _P]
_o.oracle_count.argtypes = [C.c_int64, _P, _P, C.c_int, _P, _P, C.c_int, _P]
_o.oracle_brute.argtypes = [C.c_int64, _P, _P, _P, _P, C.c_int]
_o.oracle_tomita.argtypes = [C.c_int64, _P, _P, _P, _P, C.c_int]
HIST = 4096


def _p(a):
    return a.ctypes.data_as(_P)


def _csr(g):
    rp = np.ascontiguousarray(g.row_ptr[:g.n + 1], dtype=np.int32)
    col = np.ascontiguousarray(g.col, dtype=np.int32)
    return rp, col


def peel(g):
    rp, col = _csr(g)
    prio = np.zeros(max(g.n, 1), np.uint32)
    core = np.zeros(max(g.n, 1), np.int32)
    dg = C.c_int32()
    assert _o.oracle_peel(g.n, _p(rp), _p(col), _p(prio), _p(core), C.byref(dg)) == 0
    return prio[:g.n], core[:g.n], dg.value


def orient(g, prio):
    rp, col = _csr(g)
    split = np.zeros(max(g.n, 1), np.int32)
    cs = np.zeros(max(g.m, 1), np.int32)
    pr = np.ascontiguousarray(prio, dtype=np.uint32)
    assert _o.oracle_orient(g.n, _p(rp), _p(col), _p(pr), _p(split), _p(cs)) == 0
    return split[:g.n], cs[:g.m]


def count(g, threads=0):
    """(total, hist, degeneracy) of the whole graph."""
    rp, col = _csr(g)
    tot = C.c_uint64()
    hist = np.zeros(HIST, np.uint64)
    dg = C.c_int32()
    assert _o.oracle_count(g.n, _p(rp), _p(col), threads, C.byref(tot), _p(hist), HIST,
                           C.byref(dg)) == 0
    return tot.value, hist, dg.value


def prepare(g):
    """Peel + orient: (split, cs) of the oriented CSR."""
    prio, _, _ = peel(g)
    return orient(g, prio)


def roots(g, begin=0, end=None, stride=1, threads=0, prepared=None):
    """Per-root (count, nodes) arrays plus the total over the chosen roots."""
    split, cs = prepared if prepared is not None else prepare(g)
    rp, _ = _csr(g)
    end = g.n if end is None else end
    rc = np.zeros(max(g.n, 1), np.uint64)
    rn = np.zeros(max(g.n, 1), np.uint64)
    tot = C.c_uint64()
    hist = np.zeros(HIST, np.uint64)
    assert _o.oracle_mce(g.n, _p(rp), _p(split), _p(cs), begin, end, stride, threads,
                         C.byref(tot), _p(hist), HIST, _p(rc), _p(rn)) == 0
    return tot.value, hist, rc[:g.n], rn[:g.n]


def roots_ops(g, threads=0, prepared=None):
    """Per-root (count, nodes, word ops) of every root and the total: the
    word ops are the walk's algorithmic 32-bit operations (2 W32 per row
    scored in a pivot selection + 4 W32 per tree node, W32 = ceil(d+/32))."""
    split, cs = prepared if prepared is not None else prepare(g)
    rp, _ = _csr(g)
    rc = np.zeros(max(g.n, 1), np.uint64)
    rn = np.zeros(max(g.n, 1), np.uint64)
    ro = np.zeros(max(g.n, 1), np.uint64)
    tot = C.c_uint64()
    assert _o.oracle_mce_ops(g.n, _p(rp), _p(split), _p(cs), 0, g.n, 1, threads, C.byref(tot),
                             None, 0, _p(rc), _p(rn), _p(ro)) == 0
    return tot.value, rc[:g.n], rn[:g.n], ro[:g.n]


_o.oracle_mce_l2.argtypes = [C.c_int64, _P, _P, _P, _P, C.c_int, _P, _P, C.c_int, _P, _P]


def roots_l2(g, threads=0):
    """Per-root (count, nodes) of the L2 (edge-rooted) scheme and the total:
    no pivot at the root, first-level branches in the degeneracy order."""
    prio, _, _ = peel(g)
    split, cs = orient(g, prio)
    rp, _ = _csr(g)
    pr = np.ascontiguousarray(prio, dtype=np.uint32)
    rc = np.zeros(max(g.n, 1), np.uint64)
    rn = np.zeros(max(g.n, 1), np.uint64)
    tot = C.c_uint64()
    hist = np.zeros(HIST, np.uint64)
    assert _o.oracle_mce_l2(g.n, _p(rp), _p(split), _p(cs), _p(pr), threads, C.byref(tot),
                            _p(hist), HIST, _p(rc), _p(rn)) == 0
    return tot.value, hist, rc[:g.n], rn[:g.n]


def brute(g):
    rp, col = _csr(g)
    tot = C.c_uint64()
    hist = np.zeros(HIST, np.uint64)
    assert _o.oracle_brute(g.n, _p(rp), _p(col), C.byref(tot), _p(hist), HIST) == 0
    return tot.value, hist


def tomita(g):
    rp, col = _csr(g)
    tot = C.c_uint64()
    hist = np.zeros(HIST, np.uint64)
    assert _o.oracle_tomita(g.n, _p(rp), _p(col), C.byref(tot), _p(hist), HIST) == 0
    return tot.value, hist


_o.oracle_mlp_forward.argtypes = [_P, _P, C.c_int64, _P]
_o.oracle_mlp_grad.argtypes = [_P, _P, _P, C.c_int64, _P, _P]
MLP_PARAMS = 4801


def mlp_forward(params, X):
    p = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    out = np.zeros(len(X), np.float64)
    assert _o.oracle_mlp_forward(_p(p), _p(X), len(X), _p(out)) == 0
    return out


def mlp_grad(params, X, Y):
    p = np.ascontiguousarray(params, dtype=np.float32)
    X = np.ascontiguousarray(X, dtype=np.float32)
    Y = np.ascontiguousarray(Y, dtype=np.float32)
    g = np.zeros(MLP_PARAMS, np.float64)
    loss = C.c_double()
    assert _o.oracle_mlp_grad(_p(p), _p(X), _p(Y), len(X), _p(g), C.byref(loss)) == 0
    return g, loss.value


# ---- seeded workloads, for processes that must not load libmce.so --------
class _HGraph(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int64), ("row_ptr", C.POINTER(C.c_int32)),
                ("col", C.POINTER(C.c_int32)), ("num_graphs", C.c_int32),
                ("vtx_offsets", C.POINTER(C.c_int64)), ("arc_offsets", C.POINTER(C.c_int64))]


class Graph:
    """A host CSR (row_ptr n+1, col m) with n and m, as numpy arrays."""

    def __init__(self, row_ptr, col):
        self.row_ptr, self.col = row_ptr, col
        self.n, self.m = len(row_ptr) - 1, len(col)


_o.oracle_gen_batch_union.argtypes = [C.c_int32, C.c_int64, C.c_int64, C.c_double, C.c_double,
                                      C.c_double, C.c_int32, C.c_int32, C.c_int32, C.c_uint64,
                                      C.POINTER(_HGraph), C.POINTER(C.POINTER(C.c_int64))]
_o.oracle_gen_ba.argtypes = [C.c_int64, C.c_int32, C.c_uint64, C.c_int32, C.c_int32, C.c_int32,
                             C.POINTER(_HGraph)]
_o.oracle_gen_rmat.argtypes = [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                               C.c_uint64, C.POINTER(_HGraph)]
_o.oracle_gen_er.argtypes = [C.c_int64, C.c_double, C.c_uint64, C.c_int32, C.c_int32, C.c_int32,
                             C.POINTER(_HGraph)]
_o.oracle_bel_write.argtypes = [C.c_char_p, C.POINTER(_HGraph)]
_o.oracle_hgraph_free.argtypes = [C.POINTER(_HGraph)]
_libc = C.CDLL(None)
_libc.free.argtypes = [_P]


def _take(h):
    rp = np.ctypeslib.as_array(h.row_ptr, (h.n + 1,)).copy()
    col = np.ctypeslib.as_array(h.col, (max(h.m, 1),))[:h.m].copy()
    _o.oracle_hgraph_free(C.byref(h))
    return Graph(rp, col)


def gen_batch_union(num_graphs, n_min, n_max, gamma, deg_min, deg_max, max_planted, cmin, cmax,
                    seed):
    """The disjoint union of the seeded Chung-Lu batch (the arguments of
    mce_gen_chung_lu_batch) and each graph's first union vertex."""
    h = _HGraph()
    gs = C.POINTER(C.c_int64)()
    rc = _o.oracle_gen_batch_union(num_graphs, n_min, n_max, gamma, deg_min, deg_max, max_planted,
                                   cmin, cmax, seed, C.byref(h), C.byref(gs))
    assert rc == 0, rc
    start = np.ctypeslib.as_array(gs, (num_graphs + 1,)).copy()
    _libc.free(C.cast(gs, _P))
    return _take(h), start


def gen_ba(n, m, seed, planted, cmin, cmax):
    h = _HGraph()
    assert _o.oracle_gen_ba(n, m, seed, planted, cmin, cmax, C.byref(h)) == 0
    return _take(h)


def gen_rmat(scale, ef, a, b, c, seed):
    h = _HGraph()
    assert _o.oracle_gen_rmat(scale, ef, a, b, c, seed, C.byref(h)) == 0
    return _take(h)


def gen_er(n, p, seed, planted, cmin, cmax):
    h = _HGraph()
    assert _o.oracle_gen_er(n, p, seed, planted, cmin, cmax, C.byref(h)) == 0
    return _take(h)


_o.oracle_ego_subgraph.argtypes = [_P, _P, C.c_int64, C.c_int64, C.c_int64, C.POINTER(_HGraph)]


def ego_subgraph(g, seed, cap):
    """The 2-hop ego subgraph of `seed` (mce_ego_subgraph's graph)."""
    rp, col = _csr(g)
    h = _HGraph()
    assert _o.oracle_ego_subgraph(_p(rp), _p(col), g.n, seed, cap, C.byref(h)) == 0
    return _take(h)


def bel_write(path, g):
    """Write g as a .bel file (24-byte records u64 dst, u64 src, u64 0)."""
    rp = np.ascontiguousarray(g.row_ptr[:g.n + 1], dtype=np.int32)
    col = np.ascontiguousarray(g.col, dtype=np.int32)
    vo = np.array([0, g.n + 1], np.int64)
    ao = np.array([0, g.m], np.int64)
    h = _HGraph(g.n, g.m, rp.ctypes.data_as(C.POINTER(C.c_int32)),
                col.ctypes.data_as(C.POINTER(C.c_int32)), 1,
                vo.ctypes.data_as(C.POINTER(C.c_int64)), ao.ctypes.data_as(C.POINTER(C.c_int64)))
    rc = _o.oracle_bel_write(path.encode(), C.byref(h))
    assert rc == 0, rc


def per_graph(root_counts, graph_start):
    """Per-graph sums of per-root counts over a union's vertex ranges."""
    cs = np.concatenate([[0], np.cumsum(root_counts.astype(np.uint64), dtype=np.uint64)])
    return cs[graph_start[1:]] - cs[graph_start[:-1]]
