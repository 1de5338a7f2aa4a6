"""Train the learned walk-budget MLP on the GPU and save its state.

The training graph is the lognormal-weight R-MAT stand-in for com-Orkut
(seed 2, a, b, c, d = .6, .15, .15, .1, 3,072,441 vertex ids, ~117M unique
undirected edges, weights lognormal(0, 1)).  The plain information-centric
criterion runs for a fixed number of rounds without the stop-all rule and
records every vertex's walk count (the round whose convergence check stopped
it) and mean walk length; the MLP is then trained on those labels with the
library's own kernels.

    python info-centric_ge_b200/felog_b200/train_budget.py --out budget_mlp_c4.npy

Prints one JSON line with the label distribution and the training statistics.
"""
import argparse
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import felog_b200 as fb  # noqa: E402

TRAIN = dict(size=128, window=10, negative=5, sample=1e-3, cbow=0, reuse_neg=0, min_count=0, min_rounds=2)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", required=True)
    ap.add_argument("--v-target", type=int, default=3072441)
    ap.add_argument("--e-target", type=int, default=117_000_000)
    ap.add_argument("--rounds", type=int, default=10)
    ap.add_argument("--epochs", type=int, default=6)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--seed", type=int, default=2)
    args = ap.parse_args()
    t0 = time.time()
    g = fb.synth_graph(seed=args.seed, v_target=args.v_target, e_target=args.e_target, abcd=(0.6, 0.15, 0.15, 0.1),
                       lognormal=True, holdout=0.0)
    t_graph = time.time() - t0
    V = g["v_num"]
    f = fb.Felog(v_num=V, seed=101, precision=1, **TRAIN)
    f.load_graph(g["edges"], V)
    f.init_model()
    t1 = time.time()
    for r in range(args.rounds):
        f.walk_round(r)
        f.train_round(r)
        if r + 1 >= TRAIN["min_rounds"]:
            f.budget_check(r)
    t_label = time.time() - t1
    cnt, ln = f.budget_labels()
    st = f.mlp_train(epochs=args.epochs, batch=args.batch, lr=3e-3, seed=7)
    state = f.mlp_state()
    np.save(args.out, state)
    out = {"graph": g["info"], "v_num": V, "graph_s": round(t_graph, 1), "label_rounds": args.rounds,
           "label_s": round(t_label, 1), "count_labels": np.bincount(cnt, minlength=11)[2:].tolist(),
           "length_mean": float(ln.mean()),
           "majority_accuracy": float(np.bincount(cnt).max() / len(cnt)), "train": st}
    print(json.dumps(out), flush=True)
    f.close()


if __name__ == "__main__":
    main()
