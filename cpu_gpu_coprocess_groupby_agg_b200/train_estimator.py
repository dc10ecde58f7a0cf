"""Train the learned cardinality estimator on the GPU and store its weights.

  python -m cpu_gpu_coprocess_groupby_agg_b200.train_estimator --count 20000 \
      --out cpu_gpu_coprocess_groupby_agg_b200/estimator_weights.f32 --report report.json

Tables are drawn from the batch-workload distribution (rows log-uniform in
[2^12, 2^24], distinct ids log-uniform in [16, rows/2], Zipf s in [0, 1.5],
32/64-bit keys), labelled by the plain method's exact group count, split
90/10 into training and held-out sets; the report gives held-out q-errors of
the network and of the classical estimators carried in the features.
"""
import argparse
import json
import sys
import time
from pathlib import Path

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--count", type=int, default=20000)
    ap.add_argument("--seed", type=int, default=1234)
    ap.add_argument("--epochs", type=int, default=150)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--min-log2", type=float, default=12.0)
    ap.add_argument("--max-log2", type=float, default=24.0)
    ap.add_argument("--out", default=None)
    ap.add_argument("--report", default=None)
    ap.add_argument("--save-set", default=None, help="npz file for the generated training set")
    args = ap.parse_args(argv)

    from . import Context, estimator as E
    ctx = Context(0)
    t0 = time.time()
    X, y, shapes = E.make_training_set(ctx, args.count, seed=args.seed, min_log2=args.min_log2,
                                       max_log2=args.max_log2, log_every=max(1, args.count // 10))
    t_gen = time.time() - t0
    if args.save_set:
        np.savez_compressed(args.save_set, X=X, y=y, shapes=np.array(shapes, dtype=np.float64))
    n_tr = int(0.9 * len(y))
    t1 = time.time()
    loss = E.train(ctx, X[:n_tr], y[:n_tr], epochs=args.epochs, lr=args.lr, seed=args.seed)
    t_train = time.time() - t1
    report = {"tables": len(y), "train": n_tr, "heldout": len(y) - n_tr, "gen_s": round(t_gen, 1),
              "train_s": round(t_train, 1), "train_mse_log2": loss,
              "heldout_qerror": E.evaluate(ctx, X[n_tr:], y[n_tr:]),
              "train_qerror": E.evaluate(ctx, X[:n_tr], y[:n_tr])}
    out = Path(args.out) if args.out else E.WEIGHTS
    ctx.est_get().astype(np.float32).tofile(out)
    report["weights"] = str(out)
    text = json.dumps(report, indent=1)
    print(text)
    if args.report:
        Path(args.report).write_text(text)
    ctx.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
