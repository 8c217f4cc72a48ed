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
                   help="skip the per-graph plain-path comparison (batch workload)")
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
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu):
        self.gpu, self.rows, self.proc = gpu, [], None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            threading.Thread(target=self._read, daemon=True).start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

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


def algorithmic_bytes(g, split):
    """Bytes the search must read per launch: for each root, its row and the
    later lists (with their offsets) of every neighbour it encodes."""
    rp = g.row_ptr[:g.n + 1].astype(np.int64)
    dplus = rp[1:] - split
    deg = rp[1:] - rp[:-1]
    a = 8 + 4 * dplus                               # offsets + later list of a neighbour
    nb_sum = np.zeros(g.n, np.int64)
    nz = deg > 0
    if g.m:
        acc = np.add.reduceat(a[g.col], rp[:-1][nz])
        nb_sum[nz] = acc
    roots = dplus > 0
    search = int(np.sum(8 + 4 * deg[roots] + nb_sum[roots]))
    peel = 4 * (g.n + 1) + 4 * g.m + 8 * g.m + 12 * g.n      # rows, arcs, degree RMW, init
    orient = 4 * (g.n + 1) + 4 * g.m + 4 * g.m + 4 * g.m + 16 * g.n  # arcs, prio gather, write
    return {"search": search, "peel": peel, "orient": orient}


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return json.load(f), "measured"
    except Exception:
        return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def cpu_baseline(g, budget_s=15.0):
    """The oracle (C, OpenMP, all host cores) on a bounded sample of roots.

    Peeling and orientation run once on the whole graph; their time is
    charged in proportion to the sampled share of roots."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle
    cores = os.cpu_count() or 1
    t0 = time.perf_counter()
    prep = oracle.prepare(g)
    t_prep = time.perf_counter() - t0
    split = prep[0]
    nroots = int(np.count_nonzero(g.row_ptr[1:g.n + 1] - split))

    def sample(stride):
        t0 = time.perf_counter()
        tot = oracle.roots(g, stride=stride, threads=cores, prepared=prep)[0]
        return tot, time.perf_counter() - t0, len(range(0, g.n, stride))

    stride = 1024
    tot, dt, k = sample(stride)
    if dt < budget_s / 10:
        stride = int(min(1024, max(1, stride * dt / budget_s)))
        tot, dt, k = sample(stride)
    frac = k / max(g.n, 1)
    t = dt + t_prep * frac
    return {"value": tot / t if t > 0 else None, "unit": "maximal cliques/s", "cores": cores,
            "kind": "port",
            "sample": f"every {stride}th vertex as root ({tot} maximal cliques, {dt:.2f} s search "
                      f"+ {frac:.3f} x {t_prep:.2f} s peel/orient); {nroots} roots in the workload"}


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
        split, _ = ug.split_csr()  # for the algorithmic-byte count only
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
    total = res.total if res else dg.count(stream=sptr, **kw).total

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # ---- device-resident steps
    times, stats = [], []
    with ClockSampler(local_rank) as clk:
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
    # ---- end to end: pinned host CSR -> device -> count -> host, per step
    if hb is not None:
        rp_h, col_h, vo_h, ao_h = (torch.from_numpy(x).pin_memory() for x in mce.Batch._arrays(hb))
        h2d = sum(x.numel() * x.element_size() for x in (rp_h, col_h, vo_h, ao_h))
        # one call: the batch's parts are copied while the parts already on
        # the device are peeled and oriented
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
    e2e_times = []
    barrier()
    for _ in range(args.steps):
        flush.zero_()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        r = run_e2e()
        e1.record(stream)
        e1.synchronize()
        assert r.total == total
        e2e_times.append(e0.elapsed_time(e1))
    barrier()
    e2e_ms = sum(e2e_times) / len(e2e_times)
    e2e_path = ("mce_batch_count_host (copy of each part overlapping the peel and orientation"
                " of the parts before it)" if hb is not None
                else "mce_graph_reload + mce_count")

    # max over ranks
    if world > 1:
        step_ms, e2e_ms = max_over_ranks([step_ms, e2e_ms], "cuda")
    if rank != 0:
        dg.close()
        return None
    clocks = clk.summary()
    peaks, peak_kind = measured_peaks()
    ab = algorithmic_bytes(g, split)
    count_ms = statistics.mean(s["count_ms"] for s in stats)
    peel_ms = statistics.mean(s["peel_ms"] for s in stats)
    orient_ms = statistics.mean(s["orient_ms"] for s in stats)
    # dominant phase by device time
    phases = {"search": count_ms, "peel": peel_ms, "orient": orient_ms}
    dom = max(phases, key=phases.get)
    achieved = ab[dom] / (phases[dom] / 1e3) / 1e9
    traffic, inst = None, None
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            tj = json.load(f)
        traffic = tj.get(f"{args.workload}:{dom}")
        inst = tj.get(f"{args.workload}:search_inst")
    except Exception:
        pass
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
                       tree_nodes=stats[-1]["tree_nodes"], degeneracy=stats[-1]["degeneracy"],
                       max_later_degree=stats[-1]["max_later_degree"],
                       class_roots=stats[-1]["class_roots"][:3],
                       peel_rounds=stats[-1]["peel_rounds"],
                       peel_solo_sections=stats[-1]["peel_solo_sections"],
                       peel_split_ms={k: round(stats[-1]["peel_" + k + "_ms"], 3)
                                      for k in ("scan", "round", "wait")},
                       tasks_shared=stats[-1]["donations"],
                       settings={k: kw.get(k) for k in mce.TUNED_FIELDS},
                       tuning=tuning),
        "e2e": {"value": job_value(total, e2e_ms, world), "unit": "maximal cliques/s",
                "h2d_bytes_per_step": int(h2d),
                "d2h_bytes_per_step": int(d2h + 8 * 4096 + 64 + 8 + 4 + 128),
                "ms_per_step": e2e_ms, "path": e2e_path},
        "gpu_launches": int(sum(s["kernel_launches"] for s in stats)),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                     "algorithmic_bytes": ab[dom], "peak_source": peak_kind},
        "clocks": clocks,
    }
    if inst and clocks.get("sm_mhz"):
        # the search is issue-bound, not HBM-bound: its warp-instructions per
        # call (ncu, profiles/) over its event time, against 4 issue slots per
        # SM per cycle at the sampled clock
        sms = torch.cuda.get_device_properties(local_rank).multi_processor_count
        peak = 4 * sms * clocks["sm_mhz"] * 1e6 / 1e9
        ach = inst / (count_ms / 1e3) / 1e9
        line["roofline_issue"] = {"bound": "issue", "kernel": "search", "achieved": ach,
                                  "peak": peak, "unit": "G warp-instructions/s",
                                  "frac": ach / peak, "instructions": inst,
                                  "peak_source": "4 x SMs x sampled SM clock"}
    if not args.no_compare:  # the other root orders on the same resident graph
        cmp = {}
        for name, extra in scheds.items():
            if name == sched_used:
                continue
            kk = dict(kw, **extra)
            if name != "learned":
                kk.pop("model", None)
            dg.count(stream=sptr, **kk)
            ts = []
            for _ in range(max(2, args.steps // 2)):
                flush.zero_()
                torch.cuda.synchronize()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
                r = dg.count(stream=sptr, **kk)
                e1.record(stream)
                e1.synchronize()
                assert r.total == total, f"{name} schedule changed the count"
                ts.append(e0.elapsed_time(e1))
            ms = sum(ts) / len(ts)
            cmp[name] = {"ms_per_step": round(ms, 3), "value": total / (ms / 1e3),
                         "phases_ms": {"search": round(r.stats["count_ms"], 3),
                                       "peel": round(r.stats["peel_ms"], 3),
                                       "orient": round(r.stats["orient_ms"], 3)},
                         "tasks_shared": r.stats["donations"]}
        line["config"]["other_schedules"] = cmp
    if hb is not None and not args.no_plain:
        kw_plain = {k: v for k, v in kw.items() if k not in ("cuda_graph", "model", "sched")}
        line["config"]["plain_per_graph"] = plain_per_graph(hb, 256, stream, kw_plain)
    if not args.no_cpu_baseline and world == 1:
        try:
            line["cpu_baseline"] = cpu_baseline(g)
        except Exception as e:  # the baseline is reported, never required
            line["cpu_baseline"] = {"value": None, "error": str(e)[:200]}
    dg.close()
    return line


# ---------------------------------------------------------------------------
def serve_graph(args):
    import mce_b200 as mce
    if args.serve_graph == "ba":
        return (mce.gen_ba(4_000_000, 8, 31, 200, 20, 60),
                "Barabasi-Albert n=4e6 m=8 seed 31 + 200 planted cliques U[20,60]")
    if args.serve_graph == "cl":
        return (mce.gen_chung_lu_batch(1, 4_000_000, 4_000_000, 2.3, 8.0, 8.0, 5, 5, 40, 31).graph(0),
                "Chung-Lu n=4e6 exponent 2.3 mean degree 8 seed 31 + 5 planted cliques U[5,40]")
    return (mce.gen_rmat(args.scale, 32, 0.57, 0.19, 0.19, 31),
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
    s = mce.Serve(g, ego_cap=args.ego_cap, max_nodes=args.max_nodes)
    try:
        for w in range(args.warmup):  # short traces: first-touch of arenas and code
            seeds, arr = serve_trace(hg.n, 256, args.rate, 1000 + w)
            s.run(seeds, arr)
        with ClockSampler(local_rank) as clk:
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
            "slots": st["slots"], "arena_bytes": st["arena_bytes"], "slab_bytes": st["slab_bytes"],
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
    import mce_b200 as mce
    hg, desc = serve_graph(args)
    seeds, _ = serve_trace(hg.n, args.requests, args.rate, 31)
    tmp = tempfile.mkdtemp(prefix="mce_ref_")
    bel = os.path.join(tmp, "ego.bel")
    lat, tot, per = [], 0, 0
    sample = seeds[:args.warmup + max(args.steps, 1) * 8]
    for i, sd in enumerate(sample):
        eg, _ = mce.ego_subgraph(hg, int(sd), args.ego_cap)
        mce.bel_write(bel, eg)
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


def run_reference(args, rank, world):
    """The reference's CUDA binary (built from its own sources) on a sample."""
    if rank != 0:
        return None
    if not os.path.exists(REF_BIN):
        return {"impl": "reference", "unavailable": "oracle/_ref/parallel_mce_on_gpus not built"}
    import mce_b200 as mce
    sample_graphs = None
    if args.workload == "batch":
        sample_graphs = min(args.graphs, 1024)
        b = mce.gen_chung_lu_batch(args.graphs, 64, 16384, 2.3, 8.0, 32.0, 5, 5, 40, 11)
        # the first 1024 graphs of the same seeded batch, as one disjoint union
        vo, ao = b.vtx_offsets, b.arc_offsets
        sub = mce.HostGraph(b.row_ptr[:vo[sample_graphs]].copy(), b.col[:ao[sample_graphs]].copy(),
                            int(vo[sample_graphs] - sample_graphs), int(ao[sample_graphs]),
                            sample_graphs, vo[:sample_graphs + 1].copy(), ao[:sample_graphs + 1].copy())
        g = mce.union(sub)
        _, cfg = g, {"workload": f"chung-lu batch, first {sample_graphs} of {args.graphs} graphs "
                                 "(seed 11) as one disjoint union"}
    else:
        g, cfg, _ = make_workload(args)
    cfg.update({"n": int(g.n), "arcs": int(g.m)})
    tmp = tempfile.mkdtemp(prefix="mce_ref_")
    bel = os.path.join(tmp, "g.bel")
    mce.bel_write(bel, g)
    runs = []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        r = subprocess.run([REF_BIN, "-m", "mce", "-g", bel, "-d", "0", "-p", "l1", "-i", "p",
                            "-w", "nowl"], capture_output=True, text=True, timeout=1800)
        wall = time.perf_counter() - t0
        out = re.sub(r"\x1b\[[0-9;]*m", "", r.stdout)
        found = re.findall(r"Found (.*) maximal cliques in total", out)
        degt = re.findall(r"Degeneracy ordering time: (.*) s", out)
        cnt = re.findall(r"count time (.*) s", out)
        if r.returncode != 0 or not found or not degt or not cnt:
            return {"impl": "reference", "unavailable": f"reference run failed (rc {r.returncode}): "
                    + (r.stderr or out)[-200:].replace("\n", " ")}
        if i >= args.warmup:
            runs.append((int(found[0].replace(",", "")), float(degt[0]), float(cnt[0]), wall))
    os.remove(bel)
    os.rmdir(tmp)
    total = runs[0][0]
    dev_s = statistics.mean(d + c for _, d, c, _ in runs)
    value = total / dev_s
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "maximal cliques/s",
        "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": dev_s * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
        "data": "synthetic (seeded generators; no datasets)",
        "config": dict(cfg, maximal_cliques=total,
                       timed="reference's own timers: 'Degeneracy ordering time' + 'count time' "
                             "(-m mce -p l1 -i p -w nowl)",
                       wall_s_per_run=statistics.mean(w for *_, w in runs)),
        "cpu_baseline": {"value": value, "unit": "maximal cliques/s", "cores": os.cpu_count(),
                         "kind": "reference",
                         "sample": (f"first {sample_graphs} graphs of the batch" if sample_graphs
                                    else "whole workload")
                                   + "; the reference has no CPU implementation of the search, "
                                     "its own implementation is this CUDA binary"},
        "e2e": {"value": value, "unit": "maximal cliques/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    args = parse_args()
    rank = int(os.environ.get("RANK", 0))
    world = int(os.environ.get("WORLD_SIZE", 1))
    local_rank = int(os.environ.get("LOCAL_RANK", 0))
    if world > 1:
        import datetime
        import torch
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    try:
        if args.impl == "reference":
            line = (run_reference_serve(args, rank, world) if args.workload == "serve"
                    else run_reference(args, rank, world))
        elif args.workload == "serve":
            line = run_serve(args, rank, world, local_rank)
        else:
            line = run_mine(args, rank, world, local_rank)
        if rank == 0 and line is not None:
            print(json.dumps(line), flush=True)
    finally:
        if world > 1:
            import torch
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()
