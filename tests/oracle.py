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
