"""Leave-one-stencil-out evaluation of the learned picker, and training of
the shipped model.

    python -m ots.picker --data ots/data/sweeps_b200.json --report report.json \
        [--extra ots/data/configs_b200.json --report-sizes sizes.json] \
        [--save-model ots/data/cost_model.json]

For each held-out stencil: train the MLP on every other stencil's measured
sweep (on the GPU, ots_mlp_train), rank the held-out space, measure only the
top 10 % and keep the best measured.  Reported per stencil, as the
reference's parse-weka-results.py:19-37 does, is picked/best; beside it the
model's top-1 pick, the expected best of 10 % random picks (the method
without a model at the same measuring cost) and the space's median.
"""
import argparse
import json

import numpy as np

from . import model


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--data", required=True)
    ap.add_argument("--report")
    ap.add_argument("--save-model")
    ap.add_argument("--epochs", type=int, default=300)
    ap.add_argument("--hidden", type=int, default=64)
    ap.add_argument("--layers", type=int, default=3)
    ap.add_argument("--k-frac", type=float, default=0.10)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--extra", help="a bench --configs table: its full-size workload sweeps "
                    "join the training data, and picks are also reported per size")
    ap.add_argument("--report-sizes", help="write the per-size leave-one-out report here")
    a = ap.parse_args(argv)
    base = json.load(open(a.data))["records"]
    recs = base
    if a.extra:
        full = model.workload_records(json.load(open(a.extra)))
        recs = base + full
        if a.report_sizes:
            rs = model.leave_one_out_sizes(recs, k_frac=a.k_frac, hidden=a.hidden,
                                           layers=a.layers, epochs=a.epochs, seed=a.seed)
            for s, r in sorted(rs.items()):
                if s != "_mean":
                    print("%-26s space=%4d k=%3d picked/best=%.3f top1/best=%.3f "
                          "random-k/best=%.3f" % (s, r["space"], r["k"], r["picked_over_best"],
                                                  r["top1_over_best"], r["random_k_over_best"]))
            with open(a.report_sizes, "w") as fh:
                json.dump(rs, fh, indent=1)
    # the per-stencil report ranks one problem size's space (the sweep's)
    rep = model.leave_one_out(base, k_frac=a.k_frac, hidden=a.hidden, layers=a.layers,
                              epochs=a.epochs, seed=a.seed)
    for s, r in sorted(rep.items()):
        if s == "_mean":
            continue
        print("%-18s space=%4d k=%3d picked/best=%.3f top1/best=%.3f random-k/best=%.3f "
              "median/best=%.3f rho=%.2f" % (s, r["space"], r["k"], r["picked_over_best"],
                                             r["top1_over_best"], r["random_k_over_best"],
                                             r["median_over_best"], r["spearman"]))
    if "_mean" in rep:
        print("MEAN", json.dumps(rep["_mean"]))
    if a.report:
        with open(a.report, "w") as fh:
            json.dump(rep, fh, indent=1)
    if a.save_model:
        X, y, _, _ = model.dataset(recs)
        m = model.MLP(X.shape[1], a.hidden, a.layers, seed=a.seed)
        m.fit(X, y, epochs=a.epochs, seed=a.seed)
        with open(a.save_model, "w") as fh:
            json.dump(m.to_json(), fh)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
