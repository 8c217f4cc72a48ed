#!/usr/bin/env python3
"""Benchmark: maximal cliques per second (exact count) on one B200.

Workloads (synthetic, seeded; the reference's public datasets are not
available here):
  batch  (default) 4,096 independent Chung-Lu graphs, seed 11, n log-uniform in
         [64, 16384], exponent 2.3, mean degree U[8, 32], 0-5 planted cliques
         of size U[5, 40]; counted in one pass over their disjoint union.
  rmat   R-MAT (0.57, 0.19, 0.19, 0.05), edge factor 16, seed 7, at --scale
         (default 15).  The configuration's scale 22 is infeasible for any
         exact enumerator: the count grows 4-15x per scale step.
  ba     Barabasi-Albert n = 4,000,000, m = 8, seed 23, + 200 overlapping
         planted cliques of size U[20, 60].
  er     Erdos-Renyi G(10000, 0.002), seed 1, + 20 planted cliques U[6, 12].
  serve  a resident graph answering ego-subgraph requests (2-hop ego graph of a
         uniform random seed vertex, capped at --ego-cap vertices) arriving as a
         Poisson process at --rate requests/s; reports cliques/s and p50/p99
         latency.  --serve-graph picks the resident graph: ba (default;
         Barabasi-Albert n = 4,000,000, m = 8, seed 31, + 200 planted cliques
         U[20, 60]), cl (Chung-Lu n = 4,000,000, exponent 2.3, mean degree 8,
         seed 31) or rmat (R-MAT --scale, edge factor 32, seed 31).

One step = peel + orient + search over the whole workload with the graph
resident in HBM (`value`), or through the public API with the CSR copied
from pinned host memory and the count read back inside the timed region
(`e2e`).  `--impl reference` times the reference implementation (its CUDA
binary built from source into oracle/_ref) on the same workload.
"""
import argparse
import atexit
import contextlib
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "mce-gpu_b200"))

METRIC = "maximal cliques/s (exact count), batched+learned vs plain on 1 B200; p99 ms"
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "parallel_mce_on_gpus")


# ---- ranks (one process per GPU, replicas of the same workload) ------------
def max_over_ranks(values, device):
    """Each value's maximum over the ranks: a step takes as long as its
    slowest rank.  Without a process group, the values themselves."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if torch.distributed.is_available() and torch.distributed.is_initialized():
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return [float(x) for x in t.cpu()]


def sum_over_ranks(values, device):
    """Each value summed over the ranks (throughputs of independent replicas)."""
    import torch
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    if torch.distributed.is_available() and torch.distributed.is_initialized():
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
    return [float(x) for x in t.cpu()]


def job_value(units_per_rank, ms, world):
    """Whole-job throughput of `world` replicas that each finish
    `units_per_rank` units within `ms` (the slowest rank's time)."""
    return world * units_per_rank / (ms / 1e3)


def parse_args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["mine", "reference"], default="mine")
    p.add_argument("--workload", choices=["batch", "rmat", "ba", "er", "serve"], default="batch")
    p.add_argument("--serve-graph", choices=["ba", "cl", "rmat"], default="ba")
    p.add_argument("--ego-cap", type=int, default=16384)
    p.add_argument("--rate", type=float, default=2000.0, help="serve: Poisson arrivals per second")
    p.add_argument("--requests", type=int, default=4000, help="serve: requests per timed step")
    p.add_argument("--max-nodes", type=int, default=0, help="serve: search-node budget per request")
    p.add_argument("--small-cap", type=int, default=None,
                   help="serve: footprint bound of the 256-thread slots (0: one slot class; "
                        "default: automatic)")
    p.add_argument("--scale", type=int, default=15)
    p.add_argument("--graphs", type=int, default=4096)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--wl", choices=["on", "off"], default="on", help="subtree sharing")
    p.add_argument("--donate", type=int, default=0, help="donation threshold (0: default)")
    p.add_argument("--solo", type=int, default=0, help="peel solo frontier size (0: default)")
    p.add_argument("--after", type=int, default=0, help="donate after N nodes (0: default)")
    p.add_argument("--sched", choices=["plain", "degree", "learned"], default="degree",
                   help="root order (learned: the shipped cost model of the workload family; "
                        "the others are timed beside it unless --no-compare)")
    p.add_argument("--no-compare", action="store_true", help="skip the other schedules")
    p.add_argument("--heavy-log2", type=int, default=0,
                   help="cost schedules: roots predicted >= 2^k tree nodes run first (0: default)")
    p.add_argument("--share-log2", type=int, default=0,
                   help="learned schedule: roots predicted >= 2^k nodes share at once (0: default)")
    p.add_argument("--tune", choices=["table", "retune", "off"], default="table",
                   help="search settings: from the autotuner table (tuned and stored when the "
                        "shape class is missing), re-tuned, or the library defaults")
    p.add_argument("--tune-table", default=os.path.join(ROOT, "mce-gpu_b200", "data",
                                                        "tune_table.txt"))
    p.add_argument("--no-plain", action="store_true",
                   help="skip the plain-path comparisons (batch workload)")
    p.add_argument("--no-extras", action="store_true",
                   help="batch workload: skip the brief Barabasi-Albert and serving records")
    return p.parse_args()


# ---------------------------------------------------------------------------
def make_workload(args):
    import mce_b200 as mce
    if args.workload == "batch":
        b = mce.gen_chung_lu_batch(args.graphs, 64, 16384, 2.3, 8.0, 32.0, 5, 5, 40, 11)
        g = mce.union(b)
        cfg = {"workload": f"chung-lu batch: {args.graphs} graphs, n log-uniform [64,16384], "
                           "gamma 2.3, mean degree U[8,32], 0-5 planted cliques U[5,40], seed 11",
               "graphs": args.graphs, "path": "mce_batch_count (one union, captured search)"}
        cfg.update({"n": int(g.n), "arcs": int(g.m)})
        return g, cfg, b
    elif args.workload == "rmat":
        g = mce.gen_rmat(args.scale, 16, 0.57, 0.19, 0.19, 7)
        cfg = {"workload": f"R-MAT scale {args.scale}, edge factor 16, (0.57,0.19,0.19,0.05), seed 7"}
    elif args.workload == "ba":
        g = mce.gen_ba(4_000_000, 8, 23, 200, 20, 60)
        cfg = {"workload": "Barabasi-Albert n=4e6 m=8 seed 23 + 200 overlapping planted cliques U[20,60]"}
    else:
        g = mce.gen_er(10000, 0.002, 1, 20, 6, 12)
        cfg = {"workload": "Erdos-Renyi G(10000,0.002) seed 1 + 20 planted cliques U[6,12]"}
    cfg.update({"n": int(g.n), "arcs": int(g.m), "path": "mce_count"})
    return g, cfg, None


def plain_per_graph(hb, graphs, stream, kw):
    """The plain path for a batch: each graph its own mce_count call."""
    import torch
    import mce_b200 as mce
    tot, ms = 0, 0.0
    for i in range(min(graphs, hb.num_graphs)):
        with mce.Graph.from_host(hb.graph(i), stream=stream.cuda_stream) as dg:
            dg.count(stream=stream.cuda_stream, **kw)  # warm
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = dg.count(stream=stream.cuda_stream, **kw)
            e1.record(stream)
            e1.synchronize()
            tot += r.total
            ms += e0.elapsed_time(e1)
    return {"graphs": min(graphs, hb.num_graphs), "maximal_cliques": tot, "ms": round(ms, 3),
            "value": tot / (ms / 1e3) if ms > 0 else None}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 50 ms.  Only the
    samples taken inside `window()` (the timed steps) are kept; a window
    shorter than the sampling interval keeps the first sample after it."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None
        self.active, self.started = False, threading.Event()
        self.want_next = False  # a window closed without a sample of its own

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
            self.started.wait(5.0)  # nvidia-smi takes a moment to start sampling
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.started.set()
            if self.active or self.want_next:
                self.rows.append([x.strip() for x in line.split(",")])
                self.in_window += 1
                self.want_next = False

    @contextlib.contextmanager
    def window(self):
        self.in_window = 0
        self.active = True
        try:
            yield self
        finally:
            self.active = False
            if self.in_window == 0:
                self.want_next = True
                for _ in range(100):  # up to 1 s for the sample that ends the window
                    if not self.want_next or not self.proc:
                        break
                    time.sleep(0.01)
                self.want_next = False

    def __exit__(self, *a):
        proc, self.proc = self.proc, None
        if proc:
            proc.terminate()
            try:
                proc.wait(timeout=5)
            except Exception:
                proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows if len(r) > 8
                          for i, v in enumerate(r[5:9]) if "Active" in v and "Not" not in v})
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.rows)}


def algorithmic_bytes(g, split, cs):
    """Algorithmic bytes per call of each stage, the definitions the kernels
    are held to (n vertices, m arcs, d+ later degree, N+ later neighbours).

    stage_a (peel + orient): 4(n+1) row offsets + 4m arcs read while peeling
      + 8m degree read-modify-writes, then 4m arcs + 4m priority gathers +
      4m split-row writes + 8(n+1) split offsets = 24m + 12(n+1).
    stage_b (the search's induced-subgraph build): every root reads its
      later list and, for each later neighbour, that neighbour's later list
      and two offsets: sum_r 4 (d+(r) + sum_{v in N+(r)} d+(v)) + 8 sum_r d+(r).
    search_with_earlier_rows: what the engines read besides: each root's
      whole row and the offsets and later lists of all its neighbours
      (earlier ones too: the rows that filter leaves)."""
    rp = g.row_ptr[:g.n + 1].astype(np.int64)
    sp = split.astype(np.int64)
    dplus = rp[1:] - sp
    deg = rp[1:] - rp[:-1]
    roots = dplus > 0
    sum_all = np.zeros(g.n, np.int64)
    if g.m:
        nz = deg > 0
        sum_all[nz] = np.add.reduceat((8 + 4 * dplus)[g.col], rp[:-1][nz])
    # the later part of every split row: cs[split[v] .. rp[v+1])
    marks = np.zeros(g.m + 1, np.int64)
    np.add.at(marks, sp, 1)
    np.add.at(marks, rp[1:], -1)
    later = np.cumsum(marks)[:g.m] > 0
    owner = np.repeat(np.arange(g.n), dplus)
    nb_dplus = np.bincount(owner, weights=dplus[cs[later]].astype(np.float64), minlength=g.n)
    return {"stage_a": int(24 * g.m + 12 * (g.n + 1)),
            "stage_b": int(4 * dplus.sum() + 4 * int(round(nb_dplus.sum())) + 8 * dplus.sum()),
            "search_with_earlier_rows": int(np.sum(8 + 4 * deg[roots] + sum_all[roots]))}


def kernel_source_hash(files=None):
    """Hash of CUDA sources (all of csrc/, or the named files in it): a
    profile figure is current only while the kernels it was captured on are
    unchanged."""
    import glob
    import hashlib
    h = hashlib.sha256()
    paths = (sorted(glob.glob(os.path.join(ROOT, "mce-gpu_b200", "csrc", "*"))) if files is None
             else [os.path.join(ROOT, "mce-gpu_b200", "csrc", f) for f in sorted(files)])
    for f in paths:
        with open(f, "rb") as fh:
            h.update(os.path.basename(f).encode() + fh.read())
    return h.hexdigest()[:16]


def profile_figures(workload):
    """ncu figures committed in profiles/traffic.json for this workload,
    each kept only while the sources its kernels compile from are the ones
    it was captured on.  Returns ({figure: value}, note on what was dropped)."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            tj = json.load(f)
    except Exception:
        return {}, "no profiles/traffic.json"
    out, stale = {}, []
    for k, v in tj.items():
        if not k.startswith(workload + ":") or not isinstance(v, dict):
            continue
        name = k.split(":", 1)[1]
        if v.get("hash") == kernel_source_hash(v.get("sources")):
            out[name] = v["value"]
        else:
            stale.append(name)
    return out, (f"captured on other kernel sources: {', '.join(stale)}" if stale else None)


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def oracle_check(g, budget_s=60.0):
    """The oracle (C, OpenMP, all host cores) over every root when that fits
    the budget, else over a strided sample of roots.  Returns the timing
    record for cpu_baseline and the per-root counts (None when sampled)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    prep = oracle.prepare(g)
    t_prep = time.perf_counter() - t0
    split = prep[0]
    nroots = int(np.count_nonzero(g.row_ptr[1:g.n + 1] - split))
    t0 = time.perf_counter()
    stride = 1024
    tot, _, rc, _ = oracle.roots(g, stride=stride, threads=cores, prepared=prep)
    dt = time.perf_counter() - t0
    if dt * stride < budget_s:  # every root fits the budget
        stride = 1
        t0 = time.perf_counter()
        tot, _, rc, _ = oracle.roots(g, stride=1, threads=cores, prepared=prep)
        dt = time.perf_counter() - t0
    k = len(range(0, g.n, stride))
    frac = k / max(g.n, 1)
    t = dt + t_prep * frac
    base = {"value": tot / t if t > 0 else None, "unit": "maximal cliques/s", "cores": cores,
            "kind": "port",
            "sample": (f"every root" if stride == 1 else f"every {stride}th vertex as root")
                      + f" ({tot} maximal cliques, {dt:.2f} s search + {frac:.3f} x "
                        f"{t_prep:.2f} s peel/orient); {nroots} roots in the workload"}
    return base, (rc if stride == 1 else None), tot, stride


def timed(stream, flush, fn, steps):
    """CUDA-event times (ms) of `steps` calls of fn on `stream`, L2 flushed
    before each (outside the timed region)."""
    import torch
    ts, out = [], None
    for _ in range(steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = fn()
        e1.record(stream)
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    return ts, out


# ---------------------------------------------------------------------------
def run_mine(args, rank, world, local_rank):
    import torch
    import mce_b200 as mce
    kw = dict(worker_list=mce.WL_ON if args.wl == "on" else mce.WL_OFF,
              donate_threshold=args.donate, peel_solo_max=args.solo, donate_after=args.after,
              heavy_log2=args.heavy_log2, share_log2=args.share_log2)
    scheds = {"plain": dict(sched=mce.SCHED_PLAIN), "degree": dict(sched=mce.SCHED_DEGREE)}
    wpath = os.path.join(ROOT, "mce-gpu_b200", "data", f"cost_mlp_{args.workload}.f32")
    model = None
    if os.path.exists(wpath):
        model = mce.Model(device=local_rank)
        model.load(wpath)
        scheds["learned"] = dict(sched=mce.SCHED_LEARNED, model=model)
    sched_used = args.sched if args.sched in scheds else "degree"
    kw.update(scheds[sched_used])
    torch.cuda.set_device(local_rank)
    g, cfg, hb = make_workload(args)
    stream = torch.cuda.Stream()
    sptr = stream.cuda_stream
    flush = torch.empty(256 * 1024 * 1024, dtype=torch.uint8, device="cuda")
    with mce.Graph.from_host(g, device=local_rank, stream=sptr) as ug:
        split, cs = ug.split_csr()  # for the algorithmic-byte counts only
    if hb is not None:
        dg = mce.Batch(hb, device=local_rank, stream=sptr)
        kw = dict(kw, cuda_graph=1)
    else:
        dg = mce.Graph.from_host(g, device=local_rank, stream=sptr)
    tuning = None
    if args.tune != "off":
        tkw = {k: v for k, v in kw.items() if k != "cuda_graph"}
        tuning = dg.autotune(args.tune_table, reps=2, force=args.tune == "retune", **tkw)
        kw.update(tuning["best"])
    torch.cuda.synchronize()
    res = None
    for _ in range(args.warmup):
        res = dg.count(stream=sptr, **kw)
    first = res if res else dg.count(stream=sptr, **kw)
    total = first.total

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # ---- device-resident steps
    times, stats = [], []
    clk = ClockSampler(local_rank).__enter__()  # through the end-to-end steps
    atexit.register(clk.__exit__)
    with clk.window():
        barrier()
        for _ in range(args.steps):
            flush.zero_()  # evict L2 between steps (outside the timed region)
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            r = dg.count(stream=sptr, **kw)
            e1.record(stream)
            e1.synchronize()
            assert r.total == total, "count changed between steps"
            times.append(e0.elapsed_time(e1))
            stats.append(r.stats)
        barrier()
    step_ms = sum(times) / len(times)
    per_graph_gpu = getattr(r, "per_graph", None)
    # ---- end to end: pinned host CSR -> device -> count -> host, per step
    if hb is not None:
        rp_h, col_h, vo_h, ao_h = (torch.from_numpy(x).pin_memory() for x in mce.Batch._arrays(hb))
        h2d = sum(x.numel() * x.element_size() for x in (rp_h, col_h, vo_h, ao_h))
        run_e2e = lambda: dg.count_host(rp_h.data_ptr(), col_h.data_ptr(), vo_h.data_ptr(),
                                        ao_h.data_ptr(), hb.num_graphs, stream=sptr, **kw)
        d2h = 8 * hb.num_graphs
    else:
        rp_h = torch.from_numpy(np.ascontiguousarray(g.row_ptr[:g.n + 1])).pin_memory()
        col_h = torch.from_numpy(np.ascontiguousarray(g.col)).pin_memory()
        h2d = 4 * (g.n + 1) + 4 * g.m
        def run_e2e():
            dg.reload_ptr(rp_h.data_ptr(), col_h.data_ptr(), g.n, g.m, stream=sptr)
            return dg.count(stream=sptr, **kw)
        d2h = 0
    for _ in range(args.warmup):  # the end-to-end path's own warm-up (its first allocations)
        run_e2e()
    barrier()
    with clk.window():
        e2e_times, re2e = timed(stream, flush, run_e2e, args.steps)
    clk.__exit__()
    assert re2e.total == total
    barrier()
    e2e_ms = sum(e2e_times) / len(e2e_times)
    # this box's pinned host -> device bandwidth: one plain copy of the arcs
    # (the e2e step cannot end before its copies do)
    col_d = torch.empty_like(col_h, device="cuda")

    def copy_arcs():
        with torch.cuda.stream(stream):
            col_d.copy_(col_h, non_blocking=True)
    h2d_times, _ = timed(stream, flush, copy_arcs, 3)
    h2d_gbs = col_h.numel() * col_h.element_size() / (min(h2d_times) / 1e3) / 1e9
    del col_d
    e2e_path =("mce_batch_count_host (each part's copy overlapping the work on the parts "
                "before it)" if hb is not None else "mce_graph_reload + mce_count")

    # max over ranks
    if world > 1:
        step_ms, e2e_ms = max_over_ranks([step_ms, e2e_ms], "cuda")
    if rank != 0:
        dg.close()
        return None
    clocks = clk.summary()
    peaks, peak_kind = measured_peaks()
    ab = algorithmic_bytes(g, split, cs)
    mean = lambda k: statistics.mean(s_[k] for s_ in stats)
    count_ms, peel_ms, orient_ms = mean("count_ms"), mean("peel_ms"), mean("orient_ms")
    class_ms = [round(statistics.mean(s_["class_ms"][c] for s_ in stats), 3) for c in range(3)]
    phases = {"search": count_ms, "peel": peel_ms, "orient": orient_ms}
    # ---- the search's algorithmic word operations, from the counting
    # variants of the engines (one call outside the timed steps)
    # (the counter models the IP walk: with IPX tuned on, the IP search of the
    # same graph is timed for it separately)
    ip_kw = dict(kw, x_pivot=0)
    ops = dg.count(stream=sptr, **dict(ip_kw, count_ops=True))
    if kw.get("x_pivot"):
        _, rip = timed(stream, flush, lambda: dg.count(stream=sptr, **ip_kw), 2)
        search_ms_c, walk_c = rip.stats["count_ms"], "IP, timed apart from the IPX steps"
    else:
        rip, search_ms_c, walk_c = None, count_ms, "IP, the timed steps"
    ip_nodes = rip.stats["tree_nodes"] if rip else stats[-1]["tree_nodes"]
    assert ops.total == total and ops.stats["tree_nodes"] == ip_nodes
    word_ops = int(ops.stats["word_ops"])
    sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
    clk_hz = (clocks.get("sm_mhz") or peaks.get("sm_max_mhz", 1965.0)) * 1e6
    prof, prof_note = profile_figures(args.workload)
    hbm = peaks["hbm_gbs"]
    ach_b = ab["stage_b"] / (count_ms / 1e3) / 1e9
    line = {
        "metric": METRIC,
        "value": job_value(total, step_ms, world),
        "unit": "maximal cliques/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": step_ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32", "data": "synthetic (seeded generators; no datasets)",
        "config": dict(cfg, maximal_cliques=total, parallelism=f"replicas x{world}",
                       l2="flushed between steps (256 MiB write) and inputs larger than L2",
                       sched=sched_used, phases_ms={k: round(v, 3) for k, v in phases.items()},
                       search_class_ms={"r32": class_ms[0], "r64": class_ms[1],
                                        "wide": class_ms[2]},
                       tree_nodes=stats[-1]["tree_nodes"], degeneracy=stats[-1]["degeneracy"],
                       max_later_degree=stats[-1]["max_later_degree"],
                       class_roots=stats[-1]["class_roots"][:3],
                       peel_rounds=stats[-1]["peel_rounds"],
                       tasks_shared=stats[-1]["donations"],
                       settings={k: kw.get(k) for k in mce.TUNED_FIELDS},
                       tuning=tuning),
        "e2e": {"value": job_value(total, e2e_ms, world), "unit": "maximal cliques/s",
                "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h + 8 * 4096 + 64 + 8 + 4 + 128),
                "ms_per_step": e2e_ms, "path": e2e_path,
                "ms_steps": [round(t, 3) for t in e2e_times],
                "h2d_copy_gbs": round(h2d_gbs, 2),
                "copy_bound_ms": round(h2d / h2d_gbs / 1e6, 3)},
        "gpu_launches": int(sum(s_["kernel_launches"] for s_ in stats)),
        # the search (all engine launches of a step) against HBM by its
        # stage-B algorithmic bytes
        "roofline": {"bound": "hbm", "kernel": "search (bk_*_kernel launches of one step)",
                     "achieved": ach_b, "peak": hbm, "unit": "GB/s", "frac": ach_b / hbm,
                     "traffic": prof.get("search_dram_bytes"),
                     "traffic_note": prof_note or "ncu, profiles/traffic.json",
                     "algorithmic_bytes": ab["stage_b"], "peak_source": peak_kind,
                     "with_earlier_rows": {
                         "algorithmic_bytes": ab["search_with_earlier_rows"],
                         "frac": ab["search_with_earlier_rows"] / (count_ms / 1e3) / 1e9 / hbm}},
        # stage A: peel + orient against HBM
        "roofline_stageA": {"bound": "hbm", "kernel": "peel + orient", "unit": "GB/s",
                            "algorithmic_bytes": ab["stage_a"],
                            "achieved": ab["stage_a"] / ((peel_ms + orient_ms) / 1e3) / 1e9,
                            "peak": hbm,
                            "frac": ab["stage_a"] / ((peel_ms + orient_ms) / 1e3) / 1e9 / hbm},
        # stage C: the recursion's algorithmic 32-bit word operations over the
        # search time, against the INT32 lanes (128 per SM per clock) and
        # against AND+POPC pairs at the POPC rate (16 per SM per clock)
        "roofline_stageC": {"bound": "int32", "kernel": "search", "word_ops": word_ops,
                            "walk": walk_c, "search_ms": round(search_ms_c, 3),
                            "achieved": word_ops / (search_ms_c / 1e3) / 1e9,
                            "peak": 128 * sms * clk_hz / 1e9, "unit": "G word-ops/s",
                            "frac": word_ops / (search_ms_c / 1e3) / (128 * sms * clk_hz),
                            "frac_popc_pairs": word_ops / (search_ms_c / 1e3) / (32 * sms * clk_hz),
                            "peak_source": "128 INT32 lanes x SMs x sampled SM clock; "
                                           "popc pairs: 16 POPC + 16 AND per SM per clock"},
        "clocks": clocks,
    }
    if not args.no_compare:  # the other root orders on the same resident graph
        cmp = {}
        for name, extra in scheds.items():
            if name == sched_used:
                continue
            kk = dict(kw, **extra)
            if name != "learned":
                kk.pop("model", None)
            dg.count(stream=sptr, **kk)
            ts, rr = timed(stream, flush, lambda: dg.count(stream=sptr, **kk), max(2, args.steps // 2))
            assert rr.total == total, f"{name} schedule changed the count"
            ms = sum(ts) / len(ts)
            cmp[name] = {"ms_per_step": round(ms, 3), "value": total / (ms / 1e3),
                         "phases_ms": {"search": round(rr.stats["count_ms"], 3),
                                       "peel": round(rr.stats["peel_ms"], 3),
                                       "orient": round(rr.stats["orient_ms"], 3)},
                         "tasks_shared": rr.stats["donations"]}
        line["config"]["other_schedules"] = cmp
    if hb is not None and not args.no_plain:
        # the drop-in: one mce_count on the union of the graphs with the
        # library defaults (L1, IP, worker list, vertex order), as a user of
        # the reference's CLI would run the batch
        with mce.Graph.from_host(g, device=local_rank, stream=sptr) as ug:
            ug.count(stream=sptr)
            ts, rr = timed(stream, flush, lambda: ug.count(stream=sptr), max(3, args.steps // 4))
        assert rr.total == total, "the plain union changed the count"
        pms = sum(ts) / len(ts)
        pu = {"ms_per_step": round(pms, 3), "value": total / (pms / 1e3),
              "phases_ms": {"search": round(rr.stats["count_ms"], 3),
                            "peel": round(rr.stats["peel_ms"], 3),
                            "orient": round(rr.stats["orient_ms"], 3)},
              "path": "mce_count on the disjoint union, library defaults"}
        line["config"]["plain_union"] = pu
        learned = line["config"].get("other_schedules", {}).get("learned", {}).get("value")
        if sched_used == "learned":
            learned = line["value"]
        line["config"]["vs_plain_union"] = {
            "batched": line["value"] / pu["value"],
            "batched_learned": (learned / pu["value"]) if learned else None}
        kw_plain = {k: v for k, v in kw.items() if k not in ("cuda_graph", "model", "sched")}
        line["config"]["plain_per_graph"] = plain_per_graph(hb, 256, stream, kw_plain)
    if world == 1 and not args.no_cpu_baseline:
        # the oracle on this box's host cores: the reported CPU baseline and,
        # over every root, the check of the total and the per-graph counts
        base, rc_o, o_tot, stride = oracle_check(g)
        line["cpu_baseline"] = base
        par = {"oracle_roots": "all" if stride == 1 else f"every {stride}th"}
        if rc_o is not None:
            par["oracle_total"] = int(o_tot)
            par["total_equal"] = int(o_tot) == total
            if hb is not None:
                sys.path.insert(0, os.path.join(ROOT, "tests"))
                import oracle
                start = hb.vtx_offsets - np.arange(hb.num_graphs + 1)
                per_o = oracle.per_graph(rc_o, start)
                eq = int(np.sum(per_o == np.asarray(per_graph_gpu, np.uint64)))
                par["per_graph_equal"] = f"{eq}/{hb.num_graphs}"
        line["config"]["parity"] = par
    dg.close()
    if not args.no_extras and hb is not None:
        line["config"]["ba"] = extra_ba(args, local_rank, stream, flush, kw)
        line["serve"] = extra_serve(args, local_rank)
    return line


def extra_ba(args, local_rank, stream, flush, kw):
    """C4 in brief: the Barabasi-Albert graph (n 4e6, m 8, seed 23, 200
    planted cliques U[20,60]) counted from HBM, its total checked against
    the oracle."""
    import mce_b200 as mce
    sptr = stream.cuda_stream
    g = mce.gen_ba(4_000_000, 8, 23, 200, 20, 60)
    kk = {k: v for k, v in kw.items() if k not in ("cuda_graph", "model")}
    kk["sched"] = mce.SCHED_DEGREE
    with mce.Graph.from_host(g, device=local_rank, stream=sptr) as dg:
        try:
            kk.update(dg.autotune(args.tune_table, reps=2, force=False, **kk)["best"])
        except Exception:
            pass
        first = dg.count(stream=sptr, **kk)
        ts, rr = timed(stream, flush, lambda: dg.count(stream=sptr, **kk), max(3, args.steps // 2))
    assert rr.total == first.total
    ms = sum(ts) / len(ts)
    rec = {"workload": "Barabasi-Albert n=4e6 m=8 seed 23 + 200 overlapping planted cliques U[20,60]",
           "n": int(g.n), "arcs": int(g.m), "maximal_cliques": int(rr.total),
           "ms_per_step": round(ms, 3), "value": rr.total / (ms / 1e3),
           "phases_ms": {"search": round(rr.stats["count_ms"], 3),
                         "peel": round(rr.stats["peel_ms"], 3),
                         "orient": round(rr.stats["orient_ms"], 3)}}
    if not args.no_cpu_baseline:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle
        o_tot = oracle.count(g)[0]
        rec["parity"] = {"oracle_total": int(o_tot), "total_equal": int(o_tot) == int(rr.total)}
    return rec


def extra_serve(args, local_rank):
    """C5 in brief: ego-graph requests against a resident Barabasi-Albert
    graph (n 4e6, m 8, seed 31, 200 planted cliques) arriving as a Poisson
    process at 2,000 requests/s, two traces of 2,000 requests; host-observed
    latency from arrival to answer, and a sample of answers against the
    oracle."""
    import mce_b200 as mce
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    hg = mce.gen_ba(4_000_000, 8, 31, 200, 20, 60)
    g = mce.Graph.from_host(hg, device=local_rank)
    s = mce.Serve(g, ego_cap=args.ego_cap, small_cap=args.small_cap)
    try:
        s.run(*serve_trace(hg.n, 256, 2000.0, 1000))  # first touch of the slots
        res_all, lat_all, wall = [], [], 0.0
        for k in range(2):
            seeds, arr = serve_trace(hg.n, 2000, 2000.0, 31 + k)
            t0 = time.perf_counter()
            res, lat = s.run(seeds, arr, timeout_ms=120000)
            wall += time.perf_counter() - t0
            res_all.append(res)
            lat_all.append(lat)
        st = s.stats()
    finally:
        s.close()
        g.close()
    res = np.concatenate(res_all)
    lat = np.concatenate(lat_all) / 1e3
    ok = res["status"] == mce.OK
    rng = np.random.default_rng(5)
    pick = sorted(rng.choice(len(res), size=12, replace=False), key=lambda i: int(res[i]["count"]))
    checked = mism = 0
    t_or = time.perf_counter()
    for i in pick:
        if res[i]["status"] != mce.OK or time.perf_counter() - t_or > 30:
            continue
        eg, _ = mce.ego_subgraph(hg, int(res[i]["seed"]), args.ego_cap)
        checked += 1
        mism += int(oracle.count(eg)[0] != int(res[i]["count"]))
    return {"workload": "serve: resident Barabasi-Albert n=4e6 m=8 seed 31 + 200 planted cliques; "
                        f"2-hop ego graphs capped at {args.ego_cap}; Poisson 2000 req/s",
            "requests": int(len(res)), "ok": int(ok.sum()),
            "p50_ms": pct(lat, 50), "p99_ms": pct(lat, 99), "max_ms": float(lat.max()),
            "requests_per_s": len(res) / wall,
            "cliques_per_s": float(res["count"][ok].sum()) / wall,
            "slots": st["slots"], "small_slots": st["small_slots"],
            "small_cap": st["small_cap"], "peak_in_flight": st["peak_in_flight"],
            "oracle_sample": {"checked": checked, "mismatches": mism}}


# ---------------------------------------------------------------------------
def serve_graph(args, gens=None):
    """The resident graph of the serving workload; `gens` = the oracle module
    builds the same graph without libmce.so (the reference arm)."""
    if gens is None:
        import mce_b200 as gens
        cl = lambda: gens.gen_chung_lu_batch(1, 4_000_000, 4_000_000, 2.3, 8.0, 8.0, 5, 5, 40,
                                             31).graph(0)
    else:
        cl = lambda: gens.gen_batch_union(1, 4_000_000, 4_000_000, 2.3, 8.0, 8.0, 5, 5, 40, 31)[0]
    if args.serve_graph == "ba":
        return (gens.gen_ba(4_000_000, 8, 31, 200, 20, 60),
                "Barabasi-Albert n=4e6 m=8 seed 31 + 200 planted cliques U[20,60]")
    if args.serve_graph == "cl":
        return (cl(), "Chung-Lu n=4e6 exponent 2.3 mean degree 8 seed 31 + 5 planted cliques U[5,40]")
    return (gens.gen_rmat(args.scale, 32, 0.57, 0.19, 0.19, 31),
            f"R-MAT scale {args.scale} edge factor 32 (0.57,0.19,0.19,0.05) seed 31")


def serve_trace(n, count, rate, seed):
    """Uniform random seed vertices and Poisson arrival times (microseconds)."""
    rng = np.random.default_rng(seed)
    seeds = rng.integers(0, n, count).astype(np.int64)
    arrival = np.cumsum(rng.exponential(1e6 / rate, count)) if rate > 0 else None
    return seeds, arrival


def log(msg):
    print(f"[{time.strftime('%H:%M:%S')}] {msg}", file=sys.stderr, flush=True)


def pct(x, q):
    return float(np.percentile(np.asarray(x, np.float64), q)) if len(x) else None


def run_serve(args, rank, world, local_rank):
    """Serving: requests against a resident graph, one session per GPU."""
    import torch
    import mce_b200 as mce
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    torch.cuda.set_device(local_rank)
    hg, desc = serve_graph(args)
    log(f"serve: resident graph n={hg.n} arcs={hg.m}")
    g = mce.Graph.from_host(hg, device=local_rank)
    s = mce.Serve(g, ego_cap=args.ego_cap, max_nodes=args.max_nodes, small_cap=args.small_cap)
    try:
        for w in range(args.warmup):  # short traces: first-touch of arenas and code
            seeds, arr = serve_trace(hg.n, 256, args.rate, 1000 + w)
            s.run(seeds, arr)
        with ClockSampler(local_rank) as clk, clk.window():
            if world > 1:
                torch.distributed.barrier()
            res_all, lat_all, makespans = [], [], []
            log("serve: warm-up done")
            for k in range(args.steps):
                seeds, arr = serve_trace(hg.n, args.requests, args.rate, 31 + 1000 * rank + k)
                t0 = time.perf_counter()
                res, lat = s.run(seeds, arr, timeout_ms=300000)
                makespans.append(time.perf_counter() - t0)
                res_all.append(res)
                lat_all.append(lat)
            if world > 1:
                torch.distributed.barrier()
        res = np.concatenate(res_all)
        lat = np.concatenate(lat_all) / 1e3  # ms
        ok = res["status"] == mce.OK
        cliques = int(res["count"][ok].sum())
        wall = sum(makespans)
        # capacity: every request of one trace admitted at once
        seeds_b, _ = serve_trace(hg.n, args.requests, 0, 77 + rank)
        t0 = time.perf_counter()
        res_b, lat_b = s.run(seeds_b, None, timeout_ms=300000)
        burst_s = time.perf_counter() - t0
        st = s.stats()
        # oracle check on a sample of the timed requests (smallest first, at
        # most about a minute of CPU time)
        log(f"serve: {len(res)} requests timed; oracle sample")
        rng = np.random.default_rng(5)
        pick = rng.choice(len(res), size=min(24, len(res)), replace=False)
        pick = sorted(pick, key=lambda i: int(res[i]["count"]))
        mism, checked, t_or = 0, 0, time.perf_counter()
        for i in pick:
            r = res[i]
            if r["status"] != mce.OK:
                continue
            if time.perf_counter() - t_or > 60:
                break
            eg, _ = mce.ego_subgraph(hg, int(r["seed"]), args.ego_cap)
            checked += 1
            mism += int(oracle.count(eg)[0] != int(r["count"]))
    finally:
        s.close()
        g.close()
    vals = [cliques / wall, wall]
    if world > 1:
        vals[0] = sum_over_ranks([vals[0]], "cuda")[0]
    if rank != 0:
        return None
    dev_ms = res["device_ns"][ok] / 1e6
    line = {
        "metric": METRIC, "value": float(vals[0]), "unit": "maximal cliques/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * wall / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded generator; uniform random seeds, Poisson arrivals)",
        "p99_ms": pct(lat, 99),
        "config": {
            "workload": f"serve: resident {desc}; 2-hop ego graphs capped at {args.ego_cap} "
                        f"vertices; Poisson {args.rate:g} req/s, {args.requests} requests per step",
            "n": int(hg.n), "arcs": int(hg.m), "requests": int(len(res)),
            "ok": int(ok.sum()), "over_limits": int((~ok).sum()),
            "maximal_cliques": cliques, "requests_per_s": len(res) / wall,
            "latency_ms": {"p50": pct(lat, 50), "p90": pct(lat, 90), "p99": pct(lat, 99),
                           "max": float(lat.max())},
            "device_ms": {"p50": pct(dev_ms, 50), "p99": pct(dev_ms, 99)},
            "slowest_1pct_phase_ms": {  # where the tail requests spend their slot time
                ph: float(np.mean(res[ph + "_ns"][ok][np.argsort(dev_ms)[-max(1, len(dev_ms) // 100):]]) / 1e6)
                for ph in ("extract", "order", "search")},
            "ego_n": {"p50": pct(res["ego_n"], 50), "max": int(res["ego_n"].max())},
            "ego_arcs": {"p50": pct(res["ego_arcs"], 50), "max": int(res["ego_arcs"].max())},
            "cliques_per_request": {"p50": pct(res["count"][ok], 50),
                                    "max": int(res["count"][ok].max()) if ok.any() else 0},
            "capacity": {"requests": len(res_b), "seconds": burst_s,
                         "requests_per_s": len(res_b) / burst_s,
                         "cliques_per_s": float(res_b["count"][res_b["status"] == mce.OK].sum())
                         / burst_s, "p99_ms": pct(lat_b / 1e3, 99)},
            "slots": st["slots"], "small_slots": st["small_slots"], "small_cap": st["small_cap"],
            "peak_in_flight": st["peak_in_flight"],
            "arena_bytes": st["arena_bytes"], "slab_bytes": st["slab_bytes"],
            "oracle_sample": {"checked": checked, "mismatches": mism},
            "parallelism": f"replicas x{world}",
        },
        "e2e": {"value": float(vals[0]), "unit": "maximal cliques/s",
                "h2d_bytes_per_step": 12 * args.requests, "d2h_bytes_per_step": 48 * args.requests,
                "note": "requests and answers cross the bus through mapped pinned memory; "
                        "latency is host-observed, from arrival to answer"},
        "gpu_launches": int(st["kernel_launches"]),
        "roofline": None,
        "clocks": clk.summary(),
    }
    return line


def run_reference_serve(args, rank, world):
    """The reference answers one ego graph per process run: a sample of the
    same trace's requests, each written as .bel and run through its binary."""
    if rank != 0:
        return None
    if not os.path.exists(REF_BIN):
        return {"impl": "reference", "unavailable": "oracle/_ref/parallel_mce_on_gpus not built"}
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle  # the seeded generators' second build: libmce.so stays unloaded
    hg, desc = serve_graph(args, gens=oracle)
    seeds, _ = serve_trace(hg.n, args.requests, args.rate, 31)
    tmp = tempfile.mkdtemp(prefix="mce_ref_")
    bel = os.path.join(tmp, "ego.bel")
    lat, tot, per = [], 0, 0
    sample = seeds[:args.warmup + max(args.steps, 1) * 8]
    for i, sd in enumerate(sample):
        eg = oracle.ego_subgraph(hg, int(sd), args.ego_cap)
        oracle.bel_write(bel, eg)
        t0 = time.perf_counter()
        r = subprocess.run([REF_BIN, "-m", "mce", "-g", bel, "-d", "0", "-p", "l1", "-i", "p",
                            "-w", "nowl"], capture_output=True, text=True, timeout=600)
        wall = time.perf_counter() - t0
        out = re.sub(r"\x1b\[[0-9;]*m", "", r.stdout)
        found = re.findall(r"Found (.*) maximal cliques in total", out)
        if r.returncode != 0 or not found:
            return {"impl": "reference", "unavailable": f"reference run failed (rc {r.returncode})"}
        if i >= args.warmup:
            lat.append(wall * 1e3)
            tot += int(found[0].replace(",", ""))
            per += 1
    os.remove(bel)
    os.rmdir(tmp)
    value = tot / (sum(lat) / 1e3)
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "maximal cliques/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sum(lat) / max(args.steps, 1), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded generator; uniform random seeds)",
        "p99_ms": pct(lat, 99),
        "config": {"workload": f"serve: resident {desc}; ego cap {args.ego_cap}; the reference "
                               "has no serving loop: each request is one run of its binary on "
                               "the ego graph (.bel), sequentially",
                   "requests": per, "maximal_cliques": tot,
                   "latency_ms": {"p50": pct(lat, 50), "p99": pct(lat, 99)}},
        "cpu_baseline": {"value": value, "unit": "maximal cliques/s", "cores": os.cpu_count(),
                         "kind": "reference", "sample": f"{per} requests of the trace"},
        "e2e": {"value": value, "unit": "maximal cliques/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def ref_workload(args):
    """The workload as a host CSR, made by the oracle library's build of the
    seeded generators: the reference arm's process never loads libmce.so.
    Returns (graph, config, graph_start or None)."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    if args.workload == "batch":
        g, start = oracle.gen_batch_union(args.graphs, 64, 16384, 2.3, 8.0, 32.0, 5, 5, 40, 11)
        cfg = {"workload": f"chung-lu batch: {args.graphs} graphs, n log-uniform [64,16384], "
                           "gamma 2.3, mean degree U[8,32], 0-5 planted cliques U[5,40], seed 11",
               "graphs": args.graphs,
               "path": "the reference binary on the batch's disjoint union as one .bel"}
    elif args.workload == "rmat":
        g, start = oracle.gen_rmat(args.scale, 16, 0.57, 0.19, 0.19, 7), None
        cfg = {"workload": f"R-MAT scale {args.scale}, edge factor 16, (0.57,0.19,0.19,0.05), seed 7"}
    elif args.workload == "ba":
        g, start = oracle.gen_ba(4_000_000, 8, 23, 200, 20, 60), None
        cfg = {"workload": "Barabasi-Albert n=4e6 m=8 seed 23 + 200 overlapping planted cliques U[20,60]"}
    else:
        g, start = oracle.gen_er(10000, 0.002, 1, 20, 6, 12), None
        cfg = {"workload": "Erdos-Renyi G(10000,0.002) seed 1 + 20 planted cliques U[6,12]"}
    cfg.update({"n": int(g.n), "arcs": int(g.m)})
    return g, cfg, start


def roomiest_tmpdir(need_bytes):
    """A scratch directory on whichever of the temp and the repository
    file systems has the most free space (the .bel of the batch is 5 GB)."""
    import shutil
    cands = [tempfile.gettempdir(), ROOT]
    best = max(cands, key=lambda d: shutil.disk_usage(d).free)
    if shutil.disk_usage(best).free < need_bytes + (1 << 30):
        raise RuntimeError(f"no room for a {need_bytes / 1e9:.1f} GB .bel")
    return tempfile.mkdtemp(prefix="mce_ref_", dir=best)


REF_LINES = {"read": r"Read graph time: (.*) s", "transfer": r"Transfer Time: (.*) s",
             "peel": r"Degeneracy ordering time: (.*) s", "orient": r"CSR Recreation time: (.*) s",
             "count": r"count time (.*) s", "found": r"Found (.*) maximal cliques in total"}


def ref_run(bel, timeout):
    """One run of the reference binary (L1, IP, no worker list); its own
    timers in seconds and the count it prints, or an error string."""
    t0 = time.perf_counter()
    try:
        r = subprocess.run([REF_BIN, "-m", "mce", "-g", bel, "-d", "0", "-p", "l1", "-i", "p",
                            "-w", "nowl"], capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return None, f"reference run exceeded {timeout} s"
    wall = time.perf_counter() - t0
    out = re.sub(r"\x1b\[[0-9;]*m", "", r.stdout)
    got = {k: re.findall(v, out) for k, v in REF_LINES.items()}
    if r.returncode != 0 or not all(got.values()):
        return None, (f"reference run failed (rc {r.returncode}): "
                      + (r.stderr or out)[-200:].replace("\n", " "))
    rec = {k: float(v[0]) for k, v in got.items() if k != "found"}
    rec["found"] = int(got["found"][0].replace(",", ""))
    rec["wall"] = wall
    return rec, None


def run_reference(args, rank, world):
    """The reference implementation - its CUDA binary, built from its own
    sources into oracle/_ref - on the same whole workload as the other arm.

    value = count / (its 'Degeneracy ordering time' + 'CSR Recreation time'
    + 'count time'): peel, orientation and search from a resident CSR, the
    phases the other arm's `value` times (its count time includes its
    scratch allocation, as in its own code).  e2e adds its 'Transfer Time'
    (host CSR -> device).  The .bel read is excluded from both.  Each run of
    the binary is one step; when a run takes long, fewer steps than asked are
    timed (steps_requested says how many were asked), so the arm ends within
    a few minutes.  The binary's count is checked against the oracle's."""
    if rank != 0:
        return None
    if not os.path.exists(REF_BIN):
        return {"impl": "reference", "unavailable": "oracle/_ref/parallel_mce_on_gpus not built"}
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    g, cfg, _ = ref_workload(args)
    tmp = roomiest_tmpdir(24 * g.m)
    bel = os.path.join(tmp, "g.bel")
    runs = []
    try:
        oracle.bel_write(bel, g)
        first, err = ref_run(bel, 1800)
        if err:
            return {"impl": "reference", "unavailable": err}
        budget_s = 150.0
        k = max(1, min(args.steps, int(budget_s / max(first["wall"], 1e-3))))
        warm = min(args.warmup, 1) - 1  # the first run above is a warm-up run
        for _ in range(max(warm, 0) + k):
            rec, err = ref_run(bel, 1800)
            if err:
                return {"impl": "reference", "unavailable": err}
            runs.append(rec)
        runs = runs[-k:]
    finally:
        if os.path.exists(bel):
            os.remove(bel)
        os.rmdir(tmp)
    total = runs[0]["found"]
    assert all(r["found"] == total for r in runs), "reference count changed between runs"
    # the oracle's count of the same graph (all host cores)
    t0 = time.perf_counter()
    o_total = oracle.count(g)[0]
    t_oracle = time.perf_counter() - t0
    dev_s = statistics.mean(r["peel"] + r["orient"] + r["count"] for r in runs)
    e2e_s = statistics.mean(r["transfer"] + r["peel"] + r["orient"] + r["count"] for r in runs)
    value = total / dev_s
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "maximal cliques/s",
        "n_gpus": 1, "steps": len(runs), "steps_requested": args.steps, "warmup": args.warmup,
        "ms_per_step": dev_s * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32", "data": "synthetic (seeded generators; no datasets)",
        "config": dict(cfg, maximal_cliques=total, same_config=True,
                       timed="reference's own timers: 'Degeneracy ordering time' + 'CSR Recreation "
                             "time' + 'count time' (-m mce -p l1 -i p -w nowl); e2e adds "
                             "'Transfer Time'",
                       phases_s={k: round(statistics.mean(r[k] for r in runs), 4)
                                 for k in ("read", "transfer", "peel", "orient", "count")},
                       wall_s_per_run=round(statistics.mean(r["wall"] for r in runs), 2),
                       parity={"oracle_total": o_total, "total_equal": o_total == total,
                               "oracle_s": round(t_oracle, 2)}),
        "cpu_baseline": {"value": value, "unit": "maximal cliques/s", "cores": os.cpu_count(),
                         "kind": "reference",
                         "sample": "the whole workload; the reference has no CPU implementation "
                                   "of the search, its own implementation is this CUDA binary"},
        "e2e": {"value": total / e2e_s, "unit": "maximal cliques/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0, "ms_per_step": e2e_s * 1e3},
    }
    return line


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if args.impl == "reference":  # rank 0 alone runs the reference; no process group
        line = (run_reference_serve(args, rank, world) if args.workload == "serve"
                else run_reference(args, rank, world))
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
            if line.get("config", {}).get("parity", {}).get("total_equal") is False:
                sys.exit(1)
        return
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.workload == "serve":
            line = run_serve(args, rank, world, local_rank)
        else:
            line = run_mine(args, rank, world, local_rank)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
            par = [line.get("config", {}).get("parity", {}),
                   line.get("config", {}).get("ba", {}).get("parity", {})]
            bad = any(p_.get("total_equal") is False for p_ in par) or any(
                p_.get("per_graph_equal", "0/0").split("/")[0] != p_.get("per_graph_equal", "0/0")
                .split("/")[1] for p_ in par if "per_graph_equal" in p_)
            if bad or line.get("serve", {}).get("oracle_sample", {}).get("mismatches"):
                print("bench: a count differs from the oracle", file=sys.stderr)
                sys.exit(1)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
