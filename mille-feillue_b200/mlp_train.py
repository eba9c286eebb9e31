"""Trains the learned per-tile precision selector (MF_MODE_MIXED_MLP) and
evaluates it against the precision rule and the FP64 solve.

Training data come from the solver itself. For each matrix of the
variable-coefficient Poisson family (grids 32^3 - 96^3, face coefficients
log-uniform over 1 - 8 decades), the library's precision rule is swept over
tolerance scales (mf_options.mixed_tau, from the default 1 upwards) and
every mixed solve is scored by its iterations to the 1e-10 true residual
(a solve that needs more than 1.1 x the default rule's iterations is cut
off there). The largest scale that still converges within that bound,
without falling back to FP64, labels every tile with the class the rule's
layout gives it at that scale (FP64 everywhere when even the default rule
fails), at both residual levels. The labels of this family do not depend
on the matrix size (the sweep ends at the same scale for every grid), so the
whole-matrix nnz feature f2 is drawn uniformly over [5, 8.5] (32^3 to beyond
256^3) in the training samples: the network learns to ignore it instead of
extrapolating from the training grids to the 128^3 evaluation matrices.
The network (6 -> 64 -> 64 -> 4) is
trained on the GPU by the library's own forward / backward / Adam kernels
(mf_mlp_train_dev) on standardized features; the standardization is folded
into the first layer so that the stored weights take the raw features.

    python mille-feillue_b200/mlp_train.py --out mille-feillue_b200/mlp_weights.bin
    python mille-feillue_b200/mlp_train.py --eval-only --eval-128 50

Needs a GPU. Prints one JSON line for the training run, one per evaluated
matrix and a summary line.
"""
import argparse
import ctypes as C
import importlib
import json
import os
import sys
import time

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
mf = importlib.import_module("mille-feillue_b200")

LEVEL_RES = [1.0, 1e-6]    # relative residual at which each level starts
SCALES = [1.0, 4.0, 16.0, 64.0, 256.0]
TOL = 1e-10
GRIDS = [32, 48, 64, 80, 96]


def family(grid, lg, seed):
    """Variable-coefficient Poisson with face coefficients log-uniform over lg decades."""
    return mf.Matrix.varpoisson3d(grid, 10.0 ** (-lg / 2), 10.0 ** (lg / 2), seed)


def solve(A, opts, maxiter=40000):
    t = mf.Tiles(A, opts)
    _, r = t.solve_cg(A.b(), tol=TOL, maxiter=maxiter, opts=opts)
    return t, r


def converged(r):
    return r["status"] == 0 and r["rel_residual_true"] <= TOL and not r["fell_back_fp64"]


def matrix_samples(A, rng, per_matrix):
    """Features and labels of one training matrix (both residual levels)."""
    t1, r1 = solve(A, mf.options(precision_mode=mf.MODE_MIXED_RULE))
    feats = t1.features()
    labels = np.zeros(len(feats), np.int32)  # FP64 when even the default rule fails
    best = None
    if converged(r1):
        best, labels = 1.0, t1.precisions()[0].astype(np.int32)
        cap = int(1.1 * r1["iterations"]) + 1
        for sc in SCALES[1:]:
            t, r = solve(A, mf.options(precision_mode=mf.MODE_MIXED_RULE, mixed_tau=sc), maxiter=cap)
            if not converged(r):
                break  # larger scales only round more
            best, labels = sc, t.precisions()[0].astype(np.int32)
    xs, ys = [], []
    for res in LEVEL_RES:
        f = feats.copy()
        f[:, 5] = np.log10(res)
        xs.append(f)
        ys.append(labels)
    x = np.concatenate(xs)
    y = np.concatenate(ys)
    if len(x) > per_matrix:
        sel = rng.choice(len(x), per_matrix, replace=False)
        x, y = x[sel], y[sel]
    return x, y, best


def init_weights(rng):
    w = np.zeros(mf.MLP_WEIGHTS, np.float32)
    w[0:384] = rng.standard_normal(384) * np.sqrt(2.0 / 6)
    w[448:4544] = rng.standard_normal(4096) * np.sqrt(2.0 / 64)
    w[4608:4864] = rng.standard_normal(256) * np.sqrt(1.0 / 64)
    return w


def train(x, y, steps, batch, lr, seed):
    import torch

    rng = np.random.default_rng(seed)
    mu = x.mean(0)
    sd = x.std(0)
    sd[sd < 1e-6] = 1.0
    xn = ((x - mu) / sd).astype(np.float32)
    perm = rng.permutation(len(x))
    xd = torch.tensor(xn[perm], device="cuda")
    yd = torch.tensor(y[perm].astype(np.int32), device="cuda")
    wd = torch.tensor(init_weights(rng), device="cuda")
    loss = C.c_float()
    rc = mf.lib().mf_mlp_train_dev(C.c_void_p(wd.data_ptr()), C.c_void_p(xd.data_ptr()),
                                   C.c_void_p(yd.data_ptr()), len(x), steps, batch, C.c_float(lr), C.byref(loss))
    if rc != 0:
        raise RuntimeError(f"mf_mlp_train_dev: {rc}")
    out = torch.zeros((len(x), 4), dtype=torch.float32, device="cuda")
    mf.lib().mf_mlp_forward_dev(C.c_void_p(wd.data_ptr()), C.c_void_p(xd.data_ptr()), len(x), 0,
                                C.c_void_p(out.data_ptr()))
    acc = float((out.argmax(1) == yd.long()).float().mean())
    w = wd.cpu().numpy().copy()
    # fold the standardization into layer 1: W1 (x - mu) / sd + b1
    W1 = w[0:384].reshape(64, 6)
    W1f = W1 / sd[None, :]
    w[384:448] = w[384:448] - W1f @ mu
    w[0:384] = W1f.reshape(-1)
    return w, float(loss.value), acc


def evaluate(cases, weights):
    """Per held-out matrix: the FP64 solve, the rule's and the network's
    mixed solves (the network's with its rule fallback), each checked by the
    FP64 true residual and by ||x - x_FP64|| / ||x_FP64||."""
    mf.set_mlp_weights(weights)
    rows = []
    for grid, lg, seed in cases:
        A = family(grid, lg, seed)
        b = A.b()
        t64 = mf.Tiles(A)
        x64, r64 = t64.solve_cg(b, tol=TOL, maxiter=40000)
        tr = mf.Tiles(A, mf.options(precision_mode=mf.MODE_MIXED_RULE))
        xr, rr = tr.solve_cg(b, tol=TOL, maxiter=40000)
        om = mf.options(precision_mode=mf.MODE_MIXED_MLP)
        om.reserved[6] = rr["iterations"]  # fall back above 1.1 x the rule's iterations
        tm = mf.Tiles(A, om)
        pred = tm.select_mlp(LEVEL_RES)[0]  # the network's level-0 classes
        xm, rm = tm.solve_cg(b, tol=TOL, maxiter=40000, opts=om)
        n64 = float(np.linalg.norm(x64))
        row = {"grid": grid, "log10_contrast": lg, "seed": seed,
               "fp64_iters": r64["iterations"], "fp64_ms": r64["time_ms"],
               "rule_iters": rr["iterations"], "rule_ms": rr["time_ms"], "rule_bytes": rr["spmv_bytes_level"][0],
               "rule_rel_residual_true": rr["rel_residual_true"],
               "rule_x_diff_vs_fp64": float(np.linalg.norm(xr - x64)) / n64,
               "mlp_iters": rm["iterations"], "mlp_ms": rm["time_ms"], "mlp_bytes": rm["spmv_bytes_level"][0],
               "mlp_fallback": rm["selector_fallback"], "mlp_rel_residual_true": rm["rel_residual_true"],
               "mlp_x_diff_vs_fp64": float(np.linalg.norm(xm - x64)) / n64,
               "rule_tile_frac": [float(v) for v in rr["tile_frac"]],
               "mlp_pred_frac": [float((pred == k).mean()) for k in range(4)]}
        rows.append(row)
        print(json.dumps(row), flush=True)
    mf.set_mlp_weights(None)
    return rows


def summarize(rows):
    return {
        "matrices": len(rows),
        "mlp_fallbacks": int(sum(r["mlp_fallback"] for r in rows)),
        "mlp_converged": int(sum(r["mlp_rel_residual_true"] <= TOL for r in rows)),
        "rule_converged": int(sum(r["rule_rel_residual_true"] <= TOL for r in rows)),
        "iters_mlp_over_rule": float(np.mean([r["mlp_iters"] / r["rule_iters"] for r in rows])),
        "bytes_mlp_over_rule": float(np.mean([r["mlp_bytes"] / r["rule_bytes"] for r in rows if r["rule_bytes"] > 0])),
        "time_mlp_over_rule": float(np.mean([r["mlp_ms"] / r["rule_ms"] for r in rows])),
        "time_rule_over_fp64": float(np.mean([r["rule_ms"] / r["fp64_ms"] for r in rows])),
        "time_mlp_over_fp64": float(np.mean([r["mlp_ms"] / r["fp64_ms"] for r in rows])),
        "max_x_diff_vs_fp64_rule": float(max(r["rule_x_diff_vs_fp64"] for r in rows)),
        "max_x_diff_vs_fp64_mlp": float(max(r["mlp_x_diff_vs_fp64"] for r in rows)),
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=mf.MLP_WEIGHTS_PATH)
    ap.add_argument("--weights", default=None)
    ap.add_argument("--eval-only", action="store_true")
    ap.add_argument("--matrices", type=int, default=2000)
    ap.add_argument("--per-matrix", type=int, default=3000)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=2048)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--eval-128", type=int, default=0, help="held-out 128^3 matrices to evaluate")
    args = ap.parse_args()
    rng = np.random.default_rng(args.seed)
    if args.eval_only:
        w = np.fromfile(args.weights or args.out, dtype="<f4")
    else:
        t0 = time.perf_counter()
        xs, ys, best = [], [], []
        for i in range(args.matrices):
            grid = GRIDS[i % len(GRIDS)]
            lg = float(rng.uniform(1.0, 8.0))
            x, y, b = matrix_samples(family(grid, lg, 1000 + i), rng, args.per_matrix)
            xs.append(x)
            ys.append(y)
            best.append(b)
        x = np.concatenate(xs)
        y = np.concatenate(ys)
        x[:, 2] = rng.uniform(5.0, 8.5, len(x)).astype(np.float32)  # size-invariant labels (module docstring)
        gen_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        w, loss, acc = train(x, y, args.steps, args.batch, args.lr, args.seed)
        train_s = time.perf_counter() - t0
        w.astype("<f4").tofile(args.out)
        print(json.dumps({"samples": int(len(x)), "class_frac": [float((y == k).mean()) for k in range(4)],
                          "best_scale_counts": {str(v): best.count(v) for v in sorted(set(best), key=str)},
                          "final_batch_loss": loss, "train_accuracy": acc,
                          "gen_s": gen_s, "train_s": train_s, "out": args.out}), flush=True)
    if args.eval_128:
        erng = np.random.default_rng(5000)  # held out: seeds and draws apart from the training set's
        cases = [(128, float(erng.uniform(1.0, 8.0)), 5000 + i) for i in range(args.eval_128)]
    else:
        cases = [(40, 1.5, 901), (40, 4.0, 902), (40, 7.0, 903), (56, 2.0, 904), (56, 5.0, 905), (64, 1.2, 906),
                 (64, 3.0, 907), (64, 6.0, 908)]
    rows = evaluate(cases, w)
    summ = summarize(rows)
    print(json.dumps({"summary": summ}), flush=True)


if __name__ == "__main__":
    main()
