"""ctypes binding of libmce.so, the B200 maximal-clique enumerator.

The library is C++/CUDA behind a C ABI (include/mce.h, include/mce_gen.h);
this module only marshals numpy arrays in and out of it.  Importing fails
loudly if the shared library has not been built: there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libmce.so")
HIST_MAX = 4096

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"libmce.so not found at {LIB_PATH}; build it with `make -C mce-gpu_b200` "
        "(or __graft_entry__.build())")
_lib = C.CDLL(LIB_PATH)

# status codes (include/mce.h)
OK, EINVAL, ENOMEM, ECUDA, EIO, EFORMAT, ELIMIT, ETIMEOUT, ENODEV, ESTATE, EAGAIN = (
    0, -1, -2, -3, -4, -5, -6, -7, -8, -9, -10)
SERVE_OVER_BUDGET, SERVE_OVER_ARCS, SERVE_TOO_WIDE = 0x20, 0x40, 0x0C
LEVEL_L1, LEVEL_L2 = 1, 2
INDUCED_P, INDUCED_PX = 1, 2
WL_OFF, WL_ON = 1, 2
SCHED_PLAIN, SCHED_DEGREE, SCHED_LEARNED = 0, 1, 2


class MceError(RuntimeError):
    def __init__(self, code: int, what: str):
        self.code = code
        msg = _lib.mce_strerror(code).decode()
        super().__init__(f"{what}: {msg} ({code})")


class _Opts(C.Structure):
    _fields_ = [("level", C.c_int32), ("induced", C.c_int32), ("worker_list", C.c_int32),
                ("sched", C.c_int32), ("bitmap_width", C.c_int32),
                ("warps_per_root", C.c_int32), ("donate_threshold", C.c_int32),
                ("log_roots", C.c_int32), ("x_pivot", C.c_int32),
                ("peel_solo_max", C.c_int32), ("donate_after", C.c_int32),
                ("cuda_graph", C.c_int32), ("heavy_log2", C.c_int32),
                ("share_log2", C.c_int32), ("warp_log", C.c_int32), ("wide_blocks", C.c_int32),
                ("wait_limit_ms", C.c_int32), ("count_ops", C.c_int32),
                ("bucket_warps_per_root", C.c_int32 * 3),
                ("bucket_donate_threshold", C.c_int32 * 3),
                ("bucket_donate_after", C.c_int32 * 3), ("stage_lists", C.c_int32),
                ("stream", C.c_void_p), ("model", C.c_void_p)]


class _Stats(C.Structure):
    _fields_ = [("peel_ms", C.c_double), ("orient_ms", C.c_double), ("count_ms", C.c_double),
                ("total_ms", C.c_double), ("degeneracy", C.c_int32),
                ("max_later_degree", C.c_int32), ("max_degree", C.c_int64),
                ("roots", C.c_int64), ("tree_nodes", C.c_uint64), ("donations", C.c_uint64),
                ("kernel_launches", C.c_int32), ("error_flags", C.c_uint32),
                ("class_roots", C.c_int64 * 8), ("peel_rounds", C.c_int64),
                ("peel_solo_sections", C.c_int64), ("peel_scan_ms", C.c_double),
                ("peel_round_ms", C.c_double), ("peel_wait_ms", C.c_double),
                ("word_ops", C.c_uint64), ("class_ms", C.c_double * 4)]


class _HGraph(C.Structure):
    _fields_ = [("n", C.c_int64), ("m", C.c_int64), ("row_ptr", C.POINTER(C.c_int32)),
                ("col", C.POINTER(C.c_int32)), ("num_graphs", C.c_int32),
                ("vtx_offsets", C.POINTER(C.c_int64)), ("arc_offsets", C.POINTER(C.c_int64))]


class _TuneResult(C.Structure):
    _fields_ = [("key", C.c_char * 48), ("best", _Opts), ("best_ms", C.c_double),
                ("default_ms", C.c_double), ("trials_run", C.c_int32), ("from_table", C.c_int32)]


TUNED_FIELDS = ("worker_list", "donate_after", "donate_threshold", "bitmap_width", "peel_solo_max",
                "wide_blocks", "x_pivot", "warps_per_root", "bucket_warps_per_root",
                "bucket_donate_threshold", "bucket_donate_after")


def _field(o, f):
    v = getattr(o, f)
    return tuple(int(x) for x in v) if isinstance(v, C.Array) else v


def _tune_dict(r: _TuneResult) -> dict:
    return {"key": r.key.decode(), "best": {f: _field(r.best, f) for f in TUNED_FIELDS},
            "best_ms": r.best_ms, "default_ms": r.default_ms, "trials_run": r.trials_run,
            "from_table": bool(r.from_table)}


def _opts_kwargs(o: "_Opts") -> dict:
    return {f: _field(o, f) for f in TUNED_FIELDS}


class _ServeOpts(C.Structure):
    _fields_ = [("ego_cap", C.c_int32), ("slots", C.c_int32), ("ring", C.c_uint32),
                ("idle_ms", C.c_int32), ("max_arcs", C.c_int64), ("max_nodes", C.c_int64),
                ("small_cap", C.c_int32), ("big_slots", C.c_int32),
                ("reserved", C.c_int64 * 2)]


class _ServeResult(C.Structure):
    _fields_ = [("count", C.c_uint64), ("seed", C.c_int64), ("status", C.c_int32),
                ("ego_n", C.c_int32), ("ego_arcs", C.c_int32), ("limits", C.c_uint32),
                ("device_ns", C.c_uint64), ("extract_ns", C.c_uint32), ("order_ns", C.c_uint32),
                ("search_ns", C.c_uint32), ("pad2", C.c_uint32)]


class _ServeStats(C.Structure):
    _fields_ = [("slots", C.c_int32), ("running", C.c_int32), ("ring", C.c_uint32),
                ("pad", C.c_uint32), ("submitted", C.c_uint64), ("served", C.c_uint64),
                ("tree_nodes", C.c_uint64), ("kernel_launches", C.c_int64),
                ("arena_bytes", C.c_uint64), ("slab_bytes", C.c_uint64), ("helps", C.c_uint64),
                ("small_slots", C.c_int32), ("small_cap", C.c_int32),
                ("peak_in_flight", C.c_uint64)]


_P = C.c_void_p
_sigs = {
    "mce_opts_default": (None, [_P]),
    "mce_strerror": (C.c_char_p, [C.c_int]),
    "mce_version": (C.c_char_p, []),
    "mce_hgraph_free": (None, [_P]),
    "mce_hgraph_from_edges": (C.c_int, [_P, _P, C.c_int64, C.c_int64, _P]),
    "mce_csr_validate": (C.c_int, [_P, _P, C.c_int64, C.c_int64]),
    "mce_bel_read": (C.c_int, [C.c_char_p, _P]),
    "mce_bel_write": (C.c_int, [C.c_char_p, _P]),
    "mce_convert_to_bel": (C.c_int, [C.c_char_p, C.c_char_p, _P, _P]),
    "mce_graph_upload": (C.c_int, [_P, _P, C.c_int64, C.c_int64, C.c_int32, _P, _P]),
    "mce_graph_reload": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int64, _P]),
    "mce_graph_free": (C.c_int, [_P]),
    "mce_bel_load": (C.c_int, [C.c_char_p, C.c_int32, _P, _P]),
    "mce_text_load": (C.c_int, [C.c_char_p, C.c_int32, _P, _P]),
    "mce_convert_to_bel_device": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int32, _P, _P, _P]),
    "mce_graph_size": (C.c_int, [_P, _P, _P]),
    "mce_degeneracy": (C.c_int, [_P, _P, _P, _P]),
    "mce_split_csr": (C.c_int, [_P, _P, _P]),
    "mce_count": (C.c_int, [_P, _P, _P, _P, _P]),
    "mce_root_log": (C.c_int, [_P, _P]),
    "mce_root_counts": (C.c_int, [_P, _P]),
    "mce_root_ops": (C.c_int, [_P, _P]),
    "mce_list": (C.c_int, [_P, _P, _P, C.c_int64, _P, C.c_int64, _P, _P]),
    "mce_warp_log": (C.c_int, [_P, _P, _P, _P, _P, C.c_int64, _P]),
    "mce_count_oriented_noalloc": (C.c_int, [_P, _P, _P, C.c_int64, _P, C.c_int64, _P, _P]),
    "mce_batch_upload": (C.c_int, [_P, _P, _P, _P, C.c_int32, C.c_int32, _P, _P]),
    "mce_batch_reload": (C.c_int, [_P, _P, _P, _P, _P, C.c_int32, _P]),
    "mce_batch_count": (C.c_int, [_P, _P, _P, _P, _P, _P]),
    "mce_batch_count_host": (C.c_int, [_P, _P, _P, _P, _P, C.c_int32, _P, _P, _P, _P, _P]),
    "mce_batch_free": (C.c_int, [_P]),
    "mce_model_create": (C.c_int, [C.c_int32, C.c_uint64, _P]),
    "mce_model_free": (C.c_int, [_P]),
    "mce_model_set": (C.c_int, [_P, _P]),
    "mce_model_get": (C.c_int, [_P, _P, _P]),
    "mce_root_features": (C.c_int, [_P, _P]),
    "mce_model_train": (C.c_int, [_P, _P, C.c_int32, C.c_int32, C.c_float, C.c_uint64, _P]),
    "mce_model_predict": (C.c_int, [_P, _P, _P]),
    "mce_model_eval": (C.c_int, [_P, _P, C.c_int64, _P]),
    "mce_model_grad": (C.c_int, [_P, _P, _P, C.c_int64, _P, _P]),
    "mce_shape_key": (C.c_int, [_P, C.c_char_p, C.c_size_t]),
    "mce_batch_shape_key": (C.c_int, [_P, C.c_char_p, C.c_size_t]),
    "mce_tune_lookup": (C.c_int, [C.c_char_p, C.c_char_p, _P]),
    "mce_autotune": (C.c_int, [_P, _P, C.c_char_p, C.c_int32, C.c_int32, _P]),
    "mce_batch_autotune": (C.c_int, [_P, _P, C.c_char_p, C.c_int32, C.c_int32, _P]),
    "mce_serve_opts_default": (None, [_P]),
    "mce_serve_open": (C.c_int, [_P, _P, _P]),
    "mce_serve_submit": (C.c_int, [_P, C.c_int64, _P]),
    "mce_serve_poll": (C.c_int, [_P, C.c_uint64, _P]),
    "mce_serve_wait": (C.c_int, [_P, C.c_uint64, C.c_int64, _P]),
    "mce_serve_run": (C.c_int, [_P, _P, _P, C.c_int64, C.c_int64, _P, _P]),
    "mce_serve_stats": (C.c_int, [_P, _P]),
    "mce_serve_close": (C.c_int, [_P]),
    "mce_gen_er": (C.c_int, [C.c_int64, C.c_double, C.c_uint64, C.c_int32, C.c_int32,
                             C.c_int32, _P]),
    "mce_gen_rmat": (C.c_int, [C.c_int32, C.c_int32, C.c_double, C.c_double, C.c_double,
                               C.c_uint64, _P]),
    "mce_gen_ba": (C.c_int, [C.c_int64, C.c_int32, C.c_uint64, C.c_int32, C.c_int32,
                             C.c_int32, _P]),
    "mce_gen_chung_lu_batch": (C.c_int, [C.c_int32, C.c_int64, C.c_int64, C.c_double,
                                         C.c_double, C.c_double, C.c_int32, C.c_int32,
                                         C.c_int32, C.c_uint64, _P]),
    "mce_gen_permute": (C.c_int, [_P, C.c_uint64, _P]),
    "mce_hgraph_union": (C.c_int, [_P, _P]),
    "mce_ego_subgraph": (C.c_int, [_P, _P, C.c_int64, C.c_int64, C.c_int64, _P, _P]),
}
for _name, (_res, _args) in _sigs.items():
    _f = getattr(_lib, _name)
    _f.restype = _res
    _f.argtypes = _args

# every entry point the C headers declare (checked by the CPU tests)
EXPORTED = tuple(_sigs)


def _check(rc: int, what: str) -> None:
    if rc != OK:
        raise MceError(rc, what)


def _ptr(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def version() -> str:
    return _lib.mce_version().decode()


# ---------------------------------------------------------------------------
# host graphs
# ---------------------------------------------------------------------------
@dataclass
class HostGraph:
    """A CSR graph (or a batch of them) in numpy arrays.

    For a batch, row_ptr / col hold every graph back to back and
    vtx_offsets / arc_offsets (num_graphs + 1 entries) locate graph g's rows
    (n_g + 1 local offsets) and arcs (local ids).
    """
    row_ptr: np.ndarray
    col: np.ndarray
    n: int
    m: int
    num_graphs: int = 1
    vtx_offsets: np.ndarray | None = None
    arc_offsets: np.ndarray | None = None

    def graph(self, g: int) -> "HostGraph":
        """Graph g of a batch as a single graph."""
        a, b = int(self.vtx_offsets[g]), int(self.vtx_offsets[g + 1])
        c, d = int(self.arc_offsets[g]), int(self.arc_offsets[g + 1])
        rp = self.row_ptr[a:b].copy()
        return HostGraph(rp, self.col[c:d].copy(), b - a - 1, d - c)

    def _as_struct(self) -> tuple[_HGraph, list]:
        keep = []
        h = _HGraph()
        h.n, h.m, h.num_graphs = self.n, self.m, self.num_graphs
        rp = np.ascontiguousarray(self.row_ptr, dtype=np.int32)
        col = np.ascontiguousarray(self.col, dtype=np.int32)
        vo = self.vtx_offsets if self.vtx_offsets is not None else np.array([0, self.n + 1], np.int64)
        ao = self.arc_offsets if self.arc_offsets is not None else np.array([0, self.m], np.int64)
        vo = np.ascontiguousarray(vo, dtype=np.int64)
        ao = np.ascontiguousarray(ao, dtype=np.int64)
        keep += [rp, col, vo, ao]
        h.row_ptr = rp.ctypes.data_as(C.POINTER(C.c_int32))
        h.col = col.ctypes.data_as(C.POINTER(C.c_int32))
        h.vtx_offsets = vo.ctypes.data_as(C.POINTER(C.c_int64))
        h.arc_offsets = ao.ctypes.data_as(C.POINTER(C.c_int64))
        return h, keep


def _take(h: _HGraph) -> HostGraph:
    """Copy a library-owned mce_hgraph_t into numpy and release it."""
    try:
        G = h.num_graphs
        nrp = h.n + G
        rp = np.ctypeslib.as_array(h.row_ptr, shape=(nrp,)).copy() if nrp > 0 else np.zeros(1, np.int32)
        col = (np.ctypeslib.as_array(h.col, shape=(h.m,)).copy() if h.m > 0
               else np.zeros(0, np.int32))
        vo = np.ctypeslib.as_array(h.vtx_offsets, shape=(G + 1,)).copy()
        ao = np.ctypeslib.as_array(h.arc_offsets, shape=(G + 1,)).copy()
        return HostGraph(rp, col, int(h.n), int(h.m), int(G), vo, ao)
    finally:
        _lib.mce_hgraph_free(C.byref(h))


def from_edges(src, dst, n: int = 0) -> HostGraph:
    s = np.ascontiguousarray(src, dtype=np.int64)
    d = np.ascontiguousarray(dst, dtype=np.int64)
    h = _HGraph()
    _check(_lib.mce_hgraph_from_edges(_ptr(s), _ptr(d), len(s), n, C.byref(h)), "from_edges")
    return _take(h)


def validate(g: HostGraph) -> int:
    rp = np.ascontiguousarray(g.row_ptr, dtype=np.int32)
    col = np.ascontiguousarray(g.col, dtype=np.int32)
    return _lib.mce_csr_validate(_ptr(rp), _ptr(col), g.n, g.m)


def gen_er(n, p, seed, planted=0, cmin=6, cmax=12) -> HostGraph:
    h = _HGraph()
    _check(_lib.mce_gen_er(n, p, seed, planted, cmin, cmax, C.byref(h)), "gen_er")
    return _take(h)


def gen_rmat(scale, edge_factor, a, b, c, seed) -> HostGraph:
    h = _HGraph()
    _check(_lib.mce_gen_rmat(scale, edge_factor, a, b, c, seed, C.byref(h)), "gen_rmat")
    return _take(h)


def gen_ba(n, m, seed, planted=0, cmin=20, cmax=60) -> HostGraph:
    h = _HGraph()
    _check(_lib.mce_gen_ba(n, m, seed, planted, cmin, cmax, C.byref(h)), "gen_ba")
    return _take(h)


def gen_chung_lu_batch(num_graphs, n_min, n_max, gamma, deg_min, deg_max, max_planted,
                       cmin, cmax, seed) -> HostGraph:
    h = _HGraph()
    _check(_lib.mce_gen_chung_lu_batch(num_graphs, n_min, n_max, gamma, deg_min, deg_max,
                                       max_planted, cmin, cmax, seed, C.byref(h)),
           "gen_chung_lu_batch")
    return _take(h)


def permute(g: HostGraph, seed: int) -> HostGraph:
    s, keep = g._as_struct()
    h = _HGraph()
    _check(_lib.mce_gen_permute(C.byref(s), seed, C.byref(h)), "permute")
    return _take(h)


def union(batch: HostGraph) -> HostGraph:
    s, keep = batch._as_struct()
    h = _HGraph()
    _check(_lib.mce_hgraph_union(C.byref(s), C.byref(h)), "union")
    return _take(h)


def ego_subgraph(g: HostGraph, seed_vertex: int, cap: int) -> tuple[HostGraph, np.ndarray]:
    rp = np.ascontiguousarray(g.row_ptr, dtype=np.int32)
    col = np.ascontiguousarray(g.col, dtype=np.int32)
    vmap = np.zeros(cap, np.int32)
    h = _HGraph()
    _check(_lib.mce_ego_subgraph(_ptr(rp), _ptr(col), g.n, seed_vertex, cap, C.byref(h),
                                 _ptr(vmap)), "ego_subgraph")
    eg = _take(h)
    return eg, vmap[:eg.n].copy()


def bel_read(path: str) -> HostGraph:
    h = _HGraph()
    _check(_lib.mce_bel_read(path.encode(), C.byref(h)), f"bel_read({path})")
    return _take(h)


def bel_write(path: str, g: HostGraph) -> None:
    s, keep = g._as_struct()
    _check(_lib.mce_bel_write(path.encode(), C.byref(s)), f"bel_write({path})")


def convert_to_bel(txt: str, bel: str, device: int | None = None) -> tuple[int, int]:
    """Text edge list -> .bel; (n, undirected edges) as the reference prints
    them.  device=None converts on the host, an index on that GPU."""
    n = C.c_int64()
    e = C.c_int64()
    if device is None:
        rc = _lib.mce_convert_to_bel(txt.encode(), bel.encode(), C.byref(n), C.byref(e))
    else:
        rc = _lib.mce_convert_to_bel_device(txt.encode(), bel.encode(), device, None,
                                            C.byref(n), C.byref(e))
    _check(rc, "convert_to_bel")
    return n.value, e.value


# ---------------------------------------------------------------------------
# device graphs
# ---------------------------------------------------------------------------
@dataclass
class CountResult:
    total: int
    hist: np.ndarray
    stats: dict


def _stats_dict(st: _Stats) -> dict:
    d = {k: getattr(st, k) for k, _ in _Stats._fields_ if k not in ("class_roots", "class_ms")}
    d["class_roots"] = list(st.class_roots)
    d["class_ms"] = list(st.class_ms)[:3]
    return d


def make_opts(*, sched=SCHED_PLAIN, bitmap_width=0, log_roots=False, level=LEVEL_L1,
              induced=INDUCED_P, worker_list=WL_ON, donate_threshold=0, x_pivot=0,
              peel_solo_max=0, donate_after=0, cuda_graph=0, heavy_log2=0, share_log2=0,
              warp_log=False, wide_blocks=0, wait_limit_ms=0, count_ops=False,
              warps_per_root=0, bucket_warps_per_root=(0, 0, 0),
              bucket_donate_threshold=(0, 0, 0), bucket_donate_after=(0, 0, 0), stage_lists=0,
              model=None, stream=None) -> _Opts:
    o = _Opts()
    _lib.mce_opts_default(C.byref(o))
    o.sched, o.bitmap_width, o.log_roots = sched, bitmap_width, int(bool(log_roots))
    o.level, o.induced, o.worker_list = level, induced, worker_list
    o.donate_threshold, o.x_pivot = donate_threshold, x_pivot
    o.peel_solo_max, o.donate_after, o.cuda_graph = peel_solo_max, donate_after, cuda_graph
    o.heavy_log2, o.share_log2, o.warp_log = heavy_log2, share_log2, int(warp_log)
    o.wide_blocks = wide_blocks
    o.wait_limit_ms = wait_limit_ms
    o.count_ops = int(bool(count_ops))
    o.warps_per_root = warps_per_root
    o.stage_lists = int(stage_lists)
    for i in range(3):
        o.bucket_warps_per_root[i] = int(bucket_warps_per_root[i])
        o.bucket_donate_threshold[i] = int(bucket_donate_threshold[i])
        o.bucket_donate_after[i] = int(bucket_donate_after[i])
    o.stream = stream
    o.model = model._h if model is not None else None
    return o


class Graph:
    """A graph resident on one GPU (wraps mce_graph_t)."""

    def __init__(self, row_ptr: np.ndarray, col: np.ndarray, device: int = 0, stream=None):
        self._h = C.c_void_p()
        self.row_ptr = np.ascontiguousarray(row_ptr, dtype=np.int32)
        self.col = np.ascontiguousarray(col, dtype=np.int32)
        self.n = len(self.row_ptr) - 1
        self.m = len(self.col)
        _check(_lib.mce_graph_upload(_ptr(self.row_ptr), _ptr(self.col), self.n, self.m,
                                     device, stream, C.byref(self._h)), "upload")

    @classmethod
    def from_host(cls, g: HostGraph, device: int = 0, stream=None) -> "Graph":
        return cls(g.row_ptr[:g.n + 1], g.col, device, stream)

    @classmethod
    def load_bel(cls, path: str, device: int = 0, stream=None) -> "Graph":
        """A .bel file read straight into device memory (mce_bel_load)."""
        self = cls.__new__(cls)
        self._h = C.c_void_p()
        _check(_lib.mce_bel_load(path.encode(), device, stream, C.byref(self._h)), "bel_load")
        self.row_ptr = self.col = None
        n, m = C.c_int64(), C.c_int64()
        _check(_lib.mce_graph_size(self._h, C.byref(n), C.byref(m)), "graph_size")
        self.n, self.m = n.value, m.value
        return self

    @classmethod
    def load_text(cls, path: str, device: int = 0, stream=None) -> "Graph":
        """A text edge list parsed, sorted and deduplicated on the device
        (mce_text_load); the graph load_bel builds from its .bel file."""
        self = cls.__new__(cls)
        self._h = C.c_void_p()
        _check(_lib.mce_text_load(path.encode(), device, stream, C.byref(self._h)), "text_load")
        self.row_ptr = self.col = None
        n, m = C.c_int64(), C.c_int64()
        _check(_lib.mce_graph_size(self._h, C.byref(n), C.byref(m)), "graph_size")
        self.n, self.m = n.value, m.value
        return self

    def reload_ptr(self, row_ptr_addr: int, col_addr: int, n: int, m: int, stream=None) -> None:
        """Re-upload from raw host addresses (e.g. pinned buffers), no copy in Python."""
        _check(_lib.mce_graph_reload(self._h, C.c_void_p(row_ptr_addr), C.c_void_p(col_addr), n,
                                     m, stream), "reload")
        self.n, self.m = n, m

    def close(self) -> None:
        if self._h:
            _lib.mce_graph_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def count(self, *, stream=None, **opts) -> CountResult:
        o = make_opts(stream=stream, **opts)
        total = C.c_uint64()
        hist = np.zeros(HIST_MAX, np.uint64)
        st = _Stats()
        _check(_lib.mce_count(self._h, C.byref(o), C.byref(total), _ptr(hist), C.byref(st)),
               "count")
        return CountResult(int(total.value), hist, _stats_dict(st))

    def shape_key(self) -> str:
        buf = C.create_string_buffer(48)
        _check(_lib.mce_shape_key(self._h, buf, 48), "shape_key")
        return buf.value.decode()

    def autotune(self, table: str | None = None, reps: int = 2, force: bool = False,
                 **opts) -> dict:
        """Tune this graph's shape class (or read it from `table`); returns the
        result with `best` = the tuned option values (pass them to count)."""
        o = make_opts(**opts)
        r = _TuneResult()
        _check(_lib.mce_autotune(self._h, C.byref(o), table.encode() if table else None, reps,
                                 int(force), C.byref(r)), "autotune")
        return _tune_dict(r)

    def degeneracy(self) -> tuple[np.ndarray, np.ndarray, int]:
        prio = np.zeros(max(self.n, 1), np.uint32)
        core = np.zeros(max(self.n, 1), np.int32)
        dg = C.c_int32()
        _check(_lib.mce_degeneracy(self._h, _ptr(prio), _ptr(core), C.byref(dg)), "degeneracy")
        return prio[:self.n], core[:self.n], int(dg.value)

    def split_csr(self) -> tuple[np.ndarray, np.ndarray]:
        split = np.zeros(max(self.n, 1), np.int32)
        cs = np.zeros(max(self.m, 1), np.int32)
        _check(_lib.mce_split_csr(self._h, _ptr(split), _ptr(cs)), "split_csr")
        return split[:self.n], cs[:self.m]

    def root_log(self) -> np.ndarray:
        out = np.zeros(max(self.n, 1), np.uint64)
        _check(_lib.mce_root_log(self._h, _ptr(out)), "root_log")
        return out[:self.n]

    def list_cliques(self, ids_cap: int = 1 << 22, cliques_cap: int = 1 << 20,
                     **opts) -> list[np.ndarray]:
        """Every maximal clique as an array of vertex ids (root first);
        grows the buffers once if the first caps are too small."""
        for _ in range(2):
            ids = np.zeros(max(ids_cap, 1), np.int32)
            off = np.zeros(cliques_cap + 1, np.int64)
            cnt, need = C.c_uint64(), C.c_int64()
            o = make_opts(**opts)
            rc = _lib.mce_list(self._h, C.byref(o), _ptr(ids), ids_cap, _ptr(off), cliques_cap,
                               C.byref(cnt), C.byref(need))
            if rc == ELIMIT:
                ids_cap, cliques_cap = max(ids_cap, need.value), max(cliques_cap, cnt.value)
                continue
            _check(rc, "list")
            k = cnt.value
            return [ids[off[i]:off[i + 1]].copy() for i in range(k)]
        raise MceError(ELIMIT, "list")

    def warp_log(self) -> dict:
        """Per search warp of the last count(warp_log=1 or 2): SM id, tree nodes,
        donations and (warp_log=2) clock cycles per phase (warps x 7)."""
        k = C.c_int64()
        _check(_lib.mce_warp_log(self._h, None, None, None, None, 0, C.byref(k)), "warp_log")
        n = max(k.value, 1)
        sm = np.zeros(n, np.uint32)
        nodes = np.zeros(n, np.uint64)
        don = np.zeros(n, np.uint64)
        cyc = np.zeros((n, 7), np.uint64)
        _check(_lib.mce_warp_log(self._h, _ptr(sm), _ptr(nodes), _ptr(don), _ptr(cyc), k.value,
                                 C.byref(k)), "warp_log")
        return {"sm": sm[:k.value], "nodes": nodes[:k.value], "donations": don[:k.value],
                "cycles": cyc[:k.value]}

    def root_counts(self) -> np.ndarray:
        out = np.zeros(max(self.n, 1), np.uint64)
        _check(_lib.mce_root_counts(self._h, _ptr(out)), "root_counts")
        return out[:self.n]

    def root_ops(self) -> np.ndarray:
        """Per-root algorithmic word operations of the last
        count(log_roots=True, count_ops=True)."""
        out = np.zeros(max(self.n, 1), np.uint64)
        _check(_lib.mce_root_ops(self._h, _ptr(out)), "root_ops")
        return out[:self.n]


@dataclass
class BatchResult:
    total: int
    per_graph: np.ndarray
    hist: np.ndarray
    stats: dict


class Batch:
    """Many graphs resident on one GPU as one disjoint union (wraps mce_batch_t)."""

    def __init__(self, hg: HostGraph, device: int = 0, stream=None):
        self._h = C.c_void_p()
        self._keep = self._arrays(hg)
        rp, col, vo, ao = self._keep
        self.num_graphs = hg.num_graphs
        _check(_lib.mce_batch_upload(_ptr(rp), _ptr(col), _ptr(vo), _ptr(ao), hg.num_graphs,
                                     device, stream, C.byref(self._h)), "batch_upload")

    @staticmethod
    def _arrays(hg: HostGraph):
        vo = hg.vtx_offsets if hg.vtx_offsets is not None else np.array([0, hg.n + 1], np.int64)
        ao = hg.arc_offsets if hg.arc_offsets is not None else np.array([0, hg.m], np.int64)
        return (np.ascontiguousarray(hg.row_ptr, dtype=np.int32),
                np.ascontiguousarray(hg.col, dtype=np.int32),
                np.ascontiguousarray(vo, dtype=np.int64), np.ascontiguousarray(ao, dtype=np.int64))

    def reload_ptr(self, rp_addr, col_addr, vo_addr, ao_addr, num_graphs, stream=None) -> None:
        """Re-upload from raw host addresses (e.g. pinned buffers)."""
        _check(_lib.mce_batch_reload(self._h, C.c_void_p(rp_addr), C.c_void_p(col_addr),
                                     C.c_void_p(vo_addr), C.c_void_p(ao_addr), num_graphs,
                                     stream), "batch_reload")
        self.num_graphs = num_graphs

    def shape_key(self) -> str:
        buf = C.create_string_buffer(48)
        _check(_lib.mce_batch_shape_key(self._h, buf, 48), "batch_shape_key")
        return buf.value.decode()

    def autotune(self, table: str | None = None, reps: int = 2, force: bool = False,
                 cuda_graph=1, **opts) -> dict:
        o = make_opts(cuda_graph=cuda_graph, **opts)
        r = _TuneResult()
        _check(_lib.mce_batch_autotune(self._h, C.byref(o), table.encode() if table else None,
                                       reps, int(force), C.byref(r)), "batch_autotune")
        return _tune_dict(r)

    def count(self, *, stream=None, cuda_graph=1, **opts) -> BatchResult:
        o = make_opts(stream=stream, cuda_graph=cuda_graph, **opts)
        per = np.zeros(self.num_graphs, np.uint64)
        total = C.c_uint64()
        hist = np.zeros(HIST_MAX, np.uint64)
        st = _Stats()
        _check(_lib.mce_batch_count(self._h, C.byref(o), _ptr(per), C.byref(total), _ptr(hist),
                                    C.byref(st)), "batch_count")
        return BatchResult(int(total.value), per, hist, _stats_dict(st))

    def count_host(self, row_ptr_addr: int, col_addr: int, vo_addr: int, ao_addr: int,
                   num_graphs: int, *, stream=None, cuda_graph=1, **opts) -> BatchResult:
        """Upload from raw host addresses and count in one call
        (mce_batch_count_host): the copy of each part of the batch overlaps the
        peeling and orientation of the parts already on the device."""
        o = make_opts(stream=stream, cuda_graph=cuda_graph, **opts)
        per = np.zeros(num_graphs, np.uint64)
        total = C.c_uint64()
        hist = np.zeros(HIST_MAX, np.uint64)
        st = _Stats()
        _check(_lib.mce_batch_count_host(self._h, C.c_void_p(row_ptr_addr), C.c_void_p(col_addr),
                                         C.c_void_p(vo_addr), C.c_void_p(ao_addr), num_graphs,
                                         C.byref(o), _ptr(per), C.byref(total), _ptr(hist),
                                         C.byref(st)), "batch_count_host")
        self.num_graphs = num_graphs
        return BatchResult(int(total.value), per, hist, _stats_dict(st))

    def close(self) -> None:
        if self._h:
            _lib.mce_batch_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


MLP_INPUTS, MLP_HIDDEN, MLP_PARAMS = 8, 64, 4801


class Model:
    """The cost MLP (wraps mce_model_t)."""

    def __init__(self, device: int = 0, seed: int = 1):
        self._h = C.c_void_p()
        _check(_lib.mce_model_create(device, seed, C.byref(self._h)), "model_create")

    def set(self, params: np.ndarray) -> None:
        p = np.ascontiguousarray(params, dtype=np.float32)
        assert p.size == MLP_PARAMS
        _check(_lib.mce_model_set(self._h, _ptr(p)), "model_set")

    def get(self) -> tuple[np.ndarray, np.ndarray]:
        p = np.zeros(MLP_PARAMS, np.float32)
        h = np.zeros(MLP_PARAMS, np.uint16)
        _check(_lib.mce_model_get(self._h, _ptr(p), _ptr(h)), "model_get")
        return p, h.view(np.float16)

    def save(self, path: str) -> None:
        self.get()[0].tofile(path)

    def load(self, path: str) -> None:
        self.set(np.fromfile(path, dtype=np.float32))

    def train(self, g: "Graph", epochs=8, batch=1024, lr=2e-3, seed=7) -> np.ndarray:
        loss = np.zeros(epochs, np.float32)
        _check(_lib.mce_model_train(self._h, g._h, epochs, batch, lr, seed, _ptr(loss)),
               "model_train")
        return loss

    def predict(self, g: "Graph") -> np.ndarray:
        out = np.zeros(max(g.n, 1), np.float32)
        _check(_lib.mce_model_predict(self._h, g._h, _ptr(out)), "model_predict")
        return out[:g.n]

    def eval(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.zeros(len(X), np.float32)
        _check(_lib.mce_model_eval(self._h, _ptr(X), len(X), _ptr(out)), "model_eval")
        return out

    def grad(self, X: np.ndarray, Y: np.ndarray) -> tuple[np.ndarray, float]:
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        g = np.zeros(MLP_PARAMS, np.float32)
        loss = C.c_float()
        _check(_lib.mce_model_grad(self._h, _ptr(X), _ptr(Y), len(X), _ptr(g), C.byref(loss)),
               "model_grad")
        return g, float(loss.value)

    def close(self) -> None:
        if self._h:
            _lib.mce_model_free(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def root_features(g: "Graph") -> np.ndarray:
    out = np.zeros((max(g.n, 1), MLP_INPUTS), np.float32)
    _check(_lib.mce_root_features(g._h, _ptr(out)), "root_features")
    return out[:g.n]


# ---------------------------------------------------------------------------
# serving
# ---------------------------------------------------------------------------
SERVE_RESULT_DTYPE = np.dtype([("count", np.uint64), ("seed", np.int64), ("status", np.int32),
                               ("ego_n", np.int32), ("ego_arcs", np.int32), ("limits", np.uint32),
                               ("device_ns", np.uint64), ("extract_ns", np.uint32),
                               ("order_ns", np.uint32), ("search_ns", np.uint32),
                               ("pad2", np.uint32)])
assert SERVE_RESULT_DTYPE.itemsize == C.sizeof(_ServeResult)


def _result_dict(r: _ServeResult) -> dict:
    return {k: getattr(r, k) for k, _ in _ServeResult._fields_ if k != "pad2"}


class Serve:
    """A serving session over a resident Graph (wraps mce_serve_t).

    Each request is a seed vertex; its answer is the maximal-clique count of
    the seed's 2-hop ego subgraph (ego_subgraph(host_graph, seed, ego_cap)).
    small_cap (None: automatic) routes the requests whose footprint bound
    fits it to 256-thread slots, four per block; big_slots whole-block slots
    take the others (0: half the blocks).  Request ids carry their class in
    bit 0.
    """

    def __init__(self, g: Graph, *, ego_cap=1024, slots=0, ring=4096, idle_ms=1000, max_arcs=0,
                 max_nodes=0, small_cap=None, big_slots=0):
        o = _ServeOpts()
        _lib.mce_serve_opts_default(C.byref(o))
        o.ego_cap, o.slots, o.ring, o.idle_ms = ego_cap, slots, ring, idle_ms
        o.max_arcs, o.max_nodes = max_arcs, max_nodes
        o.small_cap = -1 if small_cap is None else small_cap
        o.big_slots = big_slots
        self._h = C.c_void_p()
        self.graph = g  # the session reads the graph's device arrays
        _check(_lib.mce_serve_open(g._h, C.byref(o), C.byref(self._h)), "serve_open")

    def submit(self, seed: int) -> int:
        rid = C.c_uint64()
        _check(_lib.mce_serve_submit(self._h, seed, C.byref(rid)), "serve_submit")
        return int(rid.value)

    def poll(self, rid: int) -> dict | None:
        r = _ServeResult()
        rc = _lib.mce_serve_poll(self._h, rid, C.byref(r))
        if rc == EAGAIN:
            return None
        _check(rc, "serve_poll")
        return _result_dict(r)

    def wait(self, rid: int, timeout_ms: int = 60000) -> dict:
        r = _ServeResult()
        _check(_lib.mce_serve_wait(self._h, rid, timeout_ms, C.byref(r)), "serve_wait")
        return _result_dict(r)

    def run(self, seeds, arrival_us=None, timeout_ms: int = 600000):
        """Open-loop trace; returns (results structured array, latency_us array)."""
        seeds = np.ascontiguousarray(seeds, dtype=np.int64)
        arr = None if arrival_us is None else np.ascontiguousarray(arrival_us, dtype=np.float64)
        res = np.zeros(len(seeds), SERVE_RESULT_DTYPE)
        lat = np.zeros(len(seeds), np.float64)
        _check(_lib.mce_serve_run(self._h, _ptr(seeds), _ptr(arr), len(seeds), timeout_ms,
                                  _ptr(res), _ptr(lat)), "serve_run")
        return res, lat

    def stats(self) -> dict:
        st = _ServeStats()
        _check(_lib.mce_serve_stats(self._h, C.byref(st)), "serve_stats")
        return {k: getattr(st, k) for k, _ in _ServeStats._fields_ if k != "pad"}

    def close(self) -> None:
        if self._h:
            h, self._h = self._h, C.c_void_p()
            _check(_lib.mce_serve_close(h), "serve_close")

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()


def tune_lookup(table: str, key: str) -> dict | None:
    """The tuned option values stored for a shape class, or None."""
    o = _Opts()
    _lib.mce_opts_default(C.byref(o))
    rc = _lib.mce_tune_lookup(table.encode(), key.encode(), C.byref(o))
    if rc in (EIO, ESTATE):
        return None
    _check(rc, "tune_lookup")
    return _opts_kwargs(o)

