#!/usr/bin/env python3
"""Train the root-cost MLP for each workload family and save its weights.

Each model is trained on the GPU (this library's own forward/backward/Adam
kernels) on the search-tree sizes logged by a plain count of a graph of the
family generated with a different seed than the benchmark graph, then
checked on the benchmark-seed graph (rank correlation of predicted and true
tree sizes).  Weights: FP32 master values, MLP_PARAMS floats, in data/.

    python mce-gpu_b200/train_cost_model.py [family ...]   # ba batch rmat
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
import mce_b200 as mce  # noqa: E402

FAMILIES = {
    # family: (training graph, held-out graph = the benchmark seed)
    "ba": (lambda: mce.gen_ba(4_000_000, 8, 24, 200, 20, 60),
           lambda: mce.gen_ba(4_000_000, 8, 23, 200, 20, 60)),
    "batch": (lambda: mce.union(mce.gen_chung_lu_batch(4096, 64, 16384, 2.3, 8, 32, 5, 5, 40, 12)),
              lambda: mce.union(mce.gen_chung_lu_batch(4096, 64, 16384, 2.3, 8, 32, 5, 5, 40, 11))),
    "rmat": (lambda: mce.gen_rmat(14, 16, 0.57, 0.19, 0.19, 8),
             lambda: mce.gen_rmat(14, 16, 0.57, 0.19, 0.19, 7)),
}


def weights_path(family: str) -> str:
    return os.path.join(HERE, "data", f"cost_mlp_{family}.f32")


def rank_corr(a, b):
    ra, rb = np.argsort(np.argsort(a)), np.argsort(np.argsort(b))
    return float(np.corrcoef(ra, rb)[0, 1])


def train(family: str, epochs=8, seed=1) -> dict:
    make_train, make_test = FAMILIES[family]
    m = mce.Model(seed=seed)
    g = make_train()
    with mce.Graph.from_host(g) as dg:
        dg.count(log_roots=True)
        split, _ = dg.split_csr()
        # the model ranks roots with >= 16 later neighbours; size the run by
        # Adam steps (>= 3000) rather than by passes over few samples
        ncand = int(np.count_nonzero(g.row_ptr[1:g.n + 1] - split >= 16))
        batch = 1024 if ncand > 200_000 else 256
        epochs = max(epochs, 3000 // max(1, -(-ncand // batch)))
        losses = m.train(dg, epochs=epochs, batch=batch, lr=2e-3, seed=seed)
    with mce.Graph.from_host(make_test()) as dg:
        dg.count(log_roots=True)
        nodes = dg.root_log()
        pred = m.predict(dg)
    roots = nodes > 0
    corr = rank_corr(np.log2(1 + nodes[roots].astype(np.float64)), pred[roots])
    m.save(weights_path(family))
    return {"family": family, "samples": ncand, "epochs": epochs, "batch": batch,
            "loss_first": float(losses[0]), "loss_last": float(losses[-1]),
            "heldout_rank_corr": corr}


if __name__ == "__main__":
    for fam in (sys.argv[1:] or list(FAMILIES)):
        print(train(fam), flush=True)
