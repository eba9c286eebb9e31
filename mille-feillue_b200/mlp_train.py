"""Trains the learned per-tile precision selector (MF_MODE_MIXED_MLP) and
evaluates it against the magnitude rule and the FP64 solve.

Training data come from the solver itself. For each matrix of the
variable-coefficient Poisson family (grids and coefficient contrasts drawn
below), the magnitude rule is swept over tolerance scales
(mf_options.mixed_tau, from the default 1 upwards) and every mixed solve is
scored by its iterations to the 1e-10 true residual. The largest scale that
still converges within 10 % of the default rule's iterations, without
falling back to FP64, labels every tile at each precision level with the
rule's class at that scale (FP64 everywhere when even the default rule
fails). The network (6 -> 64 -> 64 -> 4) is trained on the GPU by the
library's own forward / backward / Adam kernels (mf_mlp_train_dev) on
standardized features; the standardization is folded into the first layer
so that the stored weights take the raw features.

    python mille-feillue_b200/mlp_train.py --out mille-feillue_b200/mlp_weights.bin
    python mille-feillue_b200/mlp_train.py --eval-only --weights mille-feillue_b200/mlp_weights.bin

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

KU = [2.0 ** -53, 2.0 ** -24, 2.0 ** -11, 2.0 ** -4]
LEVEL_TAU = [2e-7, 1e-7]   # the rule's level tolerances (precision.cu)
LEVEL_RES = [1.0, 1e-6]    # relative residual at which each level starts
SCALES = [1.0, 4.0, 16.0, 64.0, 256.0, 1024.0, 4096.0]
TOL = 1e-10


def rule(f, tau):
    """The magnitude rule (precision.cu rule_precision) on a feature array."""
    with np.errstate(over="ignore", invalid="ignore"):
        m = 10.0 ** f[:, 0].astype(np.float64)
        rng = 10.0 ** f[:, 1].astype(np.float64)
    diag = f[:, 3] > 0.5
    c = np.zeros(len(f), np.int32)
    c[KU[1] * m <= tau] = 1
    c[(~diag) & (KU[2] * m <= tau) & (rng <= 1e8)] = 2
    c[(~diag) & (KU[3] * m <= tau) & (rng <= 4096.0)] = 3
    c[~np.isfinite(m)] = 0
    return c


def family(grid, lg, seed):
    """Variable-coefficient Poisson with face coefficients log-uniform over lg decades."""
    return mf.Matrix.varpoisson3d(grid, 10.0 ** (-lg / 2), 10.0 ** (lg / 2), seed)


def solve(A, opts):
    t = mf.Tiles(A, opts)
    _, r = t.solve_cg(A.b(), tol=TOL, maxiter=40000, opts=opts)
    return t, r


def converged(r):
    return r["status"] == 0 and r["rel_residual_true"] <= TOL and not r["fell_back_fp64"]


def matrix_samples(A, rng, per_matrix):
    t1, r1 = solve(A, mf.options(precision_mode=mf.MODE_MIXED_RULE))
    feats = t1.features()
    best = None
    if converged(r1):
        best = 1.0
        for sc in SCALES[1:]:
            _, r = solve(A, mf.options(precision_mode=mf.MODE_MIXED_RULE, mixed_tau=sc))
            if converged(r) and r["iterations"] <= 1.1 * r1["iterations"]:
                best = sc
            else:
                break  # larger scales only round more
    xs, ys = [], []
    for tau, res in zip(LEVEL_TAU, LEVEL_RES):
        f = feats.copy()
        f[:, 5] = np.log10(res)
        y = rule(f, tau * best) if best is not None else np.zeros(len(f), np.int32)
        xs.append(f)
        ys.append(y)
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
    mf.set_mlp_weights(weights)
    rows = []
    for grid, lg, seed in cases:
        A = family(grid, lg, seed)
        _, r64 = solve(A, mf.options())
        _, rr = solve(A, mf.options(precision_mode=mf.MODE_MIXED_RULE))
        om = mf.options(precision_mode=mf.MODE_MIXED_MLP)
        om.reserved[6] = rr["iterations"]  # fall back above 1.1 x the rule's iterations
        tm = mf.Tiles(A, om)
        pred = tm.select_mlp(LEVEL_RES)[0]  # the network's level-0 classes
        _, rm = tm.solve_cg(A.b(), tol=TOL, maxiter=40000, opts=om)
        row = {"grid": grid, "log10_contrast": lg, "seed": seed,
               "fp64_iters": r64["iterations"], "fp64_ms": r64["time_ms"],
               "rule_iters": rr["iterations"], "rule_ms": rr["time_ms"], "rule_bytes": rr["spmv_bytes_level"][0],
               "mlp_iters": rm["iterations"], "mlp_ms": rm["time_ms"], "mlp_bytes": rm["spmv_bytes_level"][0],
               "mlp_fallback": rm["selector_fallback"], "mlp_rel_residual_true": rm["rel_residual_true"],
               "mlp_pred_frac": [float((pred == k).mean()) for k in range(4)]}
        rows.append(row)
        print(json.dumps(row), flush=True)
    mf.set_mlp_weights(None)
    return rows


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=mf.MLP_WEIGHTS_PATH)
    ap.add_argument("--weights", default=None)
    ap.add_argument("--eval-only", action="store_true")
    ap.add_argument("--matrices", type=int, default=60)
    ap.add_argument("--per-matrix", type=int, default=6000)
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--batch", type=int, default=2048)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=11)
    ap.add_argument("--eval-128", action="store_true", help="also evaluate 128^3 matrices")
    args = ap.parse_args()
    rng = np.random.default_rng(args.seed)
    if args.eval_only:
        w = np.fromfile(args.weights or args.out, dtype="<f4")
    else:
        t0 = time.perf_counter()
        xs, ys, best = [], [], []
        grids = [16, 24, 32, 40, 48]
        for i in range(args.matrices):
            grid = grids[i % len(grids)]
            lg = float(rng.uniform(1.0, 8.0))
            x, y, b = matrix_samples(family(grid, lg, 1000 + i), rng, args.per_matrix)
            xs.append(x)
            ys.append(y)
            best.append(b)
        x = np.concatenate(xs)
        y = np.concatenate(ys)
        gen_s = time.perf_counter() - t0
        t0 = time.perf_counter()
        w, loss, acc = train(x, y, args.steps, args.batch, args.lr, args.seed)
        train_s = time.perf_counter() - t0
        w.astype("<f4").tofile(args.out)
        print(json.dumps({"samples": int(len(x)), "class_frac": [float((y == k).mean()) for k in range(4)],
                          "best_scales": best, "final_batch_loss": loss, "train_accuracy": acc,
                          "gen_s": gen_s, "train_s": train_s, "out": args.out}), flush=True)
    cases = [(40, 1.5, 901), (40, 4.0, 902), (40, 7.0, 903), (56, 2.0, 904), (56, 5.0, 905), (64, 1.2, 906),
             (64, 3.0, 907), (64, 6.0, 908)]
    if args.eval_128:
        cases += [(128, 6.0, 1), (128, 2.0, 909)]
    rows = evaluate(cases, w)
    summ = {
        "matrices": len(rows),
        "mlp_fallbacks": int(sum(r["mlp_fallback"] for r in rows)),
        "mlp_converged": int(sum(r["mlp_rel_residual_true"] <= TOL for r in rows)),
        "bytes_mlp_over_rule": float(np.mean([r["mlp_bytes"] / r["rule_bytes"] for r in rows if r["rule_bytes"] > 0])),
        "time_mlp_over_rule": float(np.mean([r["mlp_ms"] / r["rule_ms"] for r in rows])),
        "time_rule_over_fp64": float(np.mean([r["rule_ms"] / r["fp64_ms"] for r in rows])),
        "time_mlp_over_fp64": float(np.mean([r["mlp_ms"] / r["fp64_ms"] for r in rows])),
    }
    print(json.dumps({"summary": summ}), flush=True)


if __name__ == "__main__":
    main()
