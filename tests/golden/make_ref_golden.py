#!/usr/bin/env python3
"""Generate tests/golden/reference_counts.json from the reference itself.

Runs the reference binary (oracle/_ref/parallel_mce_on_gpus, compiled from
the reference's own sources by `make -C oracle ref`) on seeded graphs and
records the two numbers it prints that this project must reproduce:
"Max Core = K" (the degeneracy) and "Found N maximal cliques in total.".
The reference needs a CUDA device, so this runs on the GPU machine; the
fixture it writes is committed and read by the CPU tests (pinning the
oracle) and the GPU tests (pinning the CUDA path).

Each graph is given by the generator call that makes it, so the tests can
rebuild it without storing the graph.  The reference runs with
`-p l1 -i p -w nowl`: the worker-list kernels spin until every block of a
full-GPU grid is resident, which a shared GPU does not guarantee.

It also runs `-m mce-lb-eval -p l1` and `-p l2` (no worker list) and sums
the per-block "Number of traversed nodes" lines: the search-tree sizes of
the L1 and the edge-rooted L2 schemes, which pin the oracle's trees, not
only its counts (the count does not depend on the scheme).
"""
import json
import os
import re
import subprocess
import sys
import tempfile

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "mce-gpu_b200"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import mce_b200 as mce  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "parallel_mce_on_gpus")

# name -> (generator, kwargs); kept small enough for the CPU oracle to check
GRAPHS = {
    "er_10000_0.002_s1_p20": ("gen_er", dict(n=10000, p=0.002, seed=1, planted=20, cmin=6, cmax=12)),
    "er_3000_0.01_s3_p10": ("gen_er", dict(n=3000, p=0.01, seed=3, planted=10, cmin=6, cmax=20)),
    "er_2000_0.005_s21_wide": ("gen_er", dict(n=2000, p=0.005, seed=21, planted=6, cmin=70, cmax=300)),
    "rmat_10_s7": ("gen_rmat", dict(scale=10, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=7)),
    "rmat_11_s7": ("gen_rmat", dict(scale=11, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=7)),
    "rmat_12_s7": ("gen_rmat", dict(scale=12, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=7)),
    "rmat_13_s7": ("gen_rmat", dict(scale=13, edge_factor=16, a=0.57, b=0.19, c=0.19, seed=7)),
    "ba_100000_8_s23_p40": ("gen_ba", dict(n=100000, m=8, seed=23, planted=40, cmin=20, cmax=60)),
    "chung_lu_48_s11_union": ("chung_lu_union", dict(num_graphs=48, n_min=64, n_max=16384, gamma=2.3,
                                                      deg_min=8.0, deg_max=32.0, max_planted=5,
                                                      cmin=5, cmax=40, seed=11)),
}


def make(name):
    fn, kw = GRAPHS[name]
    if fn == "chung_lu_union":
        return mce.union(mce.gen_chung_lu_batch(*kw.values()))
    return getattr(mce, fn)(*kw.values())


def run_reference(bel):
    r = subprocess.run([REF, "-m", "mce", "-g", bel, "-d", "0", "-p", "l1", "-i", "p", "-w", "nowl"],
                       capture_output=True, text=True, timeout=600)
    out = re.sub(r"\x1b\[[0-9;]*m", "", r.stdout)
    found = re.findall(r"Found (.*) maximal cliques in total", out)
    core = re.findall(r"Max Core = (-?\d+)", out)
    if r.returncode != 0 or not found or not core:
        raise RuntimeError(f"reference failed on {bel}: rc={r.returncode} {r.stderr[-300:]}")
    return int(found[0].replace(",", "")), int(core[0])


def run_lb(bel, level):
    """Total traversed nodes of the reference's -m mce-lb-eval run."""
    r = subprocess.run([REF, "-m", "mce-lb-eval", "-g", bel, "-d", "0", "-p", level, "-i", "p",
                        "-w", "nowl"], capture_output=True, text=True, timeout=600)
    out = re.sub(r"\x1b\[[0-9;]*m", "", r.stdout)
    if r.returncode != 0 or "Number of traversed nodes" not in out:
        raise RuntimeError(f"reference lb-eval failed on {bel}: rc={r.returncode}")
    body = out.split("Number of traversed nodes", 1)[1]
    return sum(int(m.group(1)) for m in re.finditer(r"^\s*\d+,\s*\d+,\s*(\d+)\s*$", body,
                                                   re.M))


def main():
    out = {}
    tmp = tempfile.mkdtemp(prefix="golden_")
    for name in GRAPHS:
        g = make(name)
        bel = os.path.join(tmp, name + ".bel")
        mce.bel_write(bel, g)
        count, core = run_reference(bel)
        nodes_l1, nodes_l2 = run_lb(bel, "l1"), run_lb(bel, "l2")
        os.remove(bel)
        out[name] = {"generator": GRAPHS[name][0], "args": GRAPHS[name][1], "n": int(g.n),
                     "arcs": int(g.m), "reference_count": count, "reference_max_core": core,
                     "reference_tree_nodes_l1": nodes_l1, "reference_tree_nodes_l2": nodes_l2}
        print(name, count, core, nodes_l1, nodes_l2, flush=True)
    dst = sys.argv[1] if len(sys.argv) > 1 else os.path.join(HERE, "reference_counts.json")
    with open(dst, "w") as f:
        json.dump({"source": "reference binary (oracle/_ref) on a B200: -m mce -p l1 -i p -w nowl "
                             "(count, max core); -m mce-lb-eval -p l1|l2 -i p -w nowl (traversed "
                             "nodes summed over blocks)",
                   "graphs": out}, f, indent=1)


if __name__ == "__main__":
    main()
