"""Runs one kernel of the solver on a fixed workload, for profilers.

  python mille-feillue_b200/prof_case.py --kernel spmv --grid 128 --reps 3
  python mille-feillue_b200/prof_case.py --kernel cg --grid 128 --iters 50
  python mille-feillue_b200/prof_case.py --kernel bicgstab --grid 64 --iters 20
  python mille-feillue_b200/prof_case.py --kernel multi --grid 128 --iters 50

spmv: `reps` launches of the tiled SpMV (k_spmv) on x*.
cg / bicgstab: one persistent-solver launch with a fixed iteration count
(0 = to the 1e-10 tolerance). multi: CG on 16 right-hand sides (U[-1, 1],
seed 0) for `iters` iterations (panel product, scalar and update kernels).
Matrix: the 3D variable-coefficient Poisson (cg, spmv, multi) or
convection-diffusion (bicgstab) of the given grid.
"""
import argparse
import importlib
import os
import sys

import numpy as np

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--kernel", default="spmv", choices=["spmv", "cg", "pcg", "bicgstab", "multi"])
    ap.add_argument("--grid", type=int, default=128)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--iters", type=int, default=50)
    ap.add_argument("--mode", default="fp64", choices=["fp64", "mixed", "fp32", "fp16", "fp8"])
    ap.add_argument("--slab-bytes", type=int, default=0)
    ap.add_argument("--rb-per-slab", type=int, default=0)
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    ap.add_argument("--time", action="store_true", help="print the CUDA-event time of the launches")
    ap.add_argument("--trace", type=int, default=0, help="trace the phases of the first N CG iterations")
    ap.add_argument("--prefetch", action="store_true", help="L2 prefetch of slabs ahead of the copy ring")
    ap.add_argument("--no-tmem", action="store_true", help="single-reduction CG with x, r in global memory")
    args = ap.parse_args()
    import torch

    mf = importlib.import_module("mille-feillue_b200")
    if args.kernel == "bicgstab":
        A = mf.Matrix.convdiff3d(args.grid)
    else:
        A = mf.Matrix.varpoisson3d(args.grid)
    if args.kernel == "multi":
        B = np.random.default_rng(0).uniform(-1, 1, (A.n, 16))
        X, it, rel, ms = mf.solve_cg_multi(A, B, tol=1e-30, maxiter=args.iters)
        print("multi 16 rhs: %d iterations %.2f ms -> %.1f us/iteration"
              % (int(it.max()), ms, ms * 1e3 / max(1, int(it.max()))))
        return
    kw = {}
    level = -1
    if args.mode == "mixed":
        kw = dict(precision_mode=mf.MODE_MIXED_RULE)
        level = 0
    elif args.mode in ("fp32", "fp16", "fp8"):
        kw = dict(precision_mode=mf.MODE_FIXED, fixed_precision={"fp32": 1, "fp16": 2, "fp8": 3}[args.mode])
        level = 0
    kw.update(slab_bytes=args.slab_bytes, rb_per_slab=args.rb_per_slab, ctas_per_sm=args.ctas_per_sm)
    opts = mf.options(**kw)
    if args.prefetch:
        opts.reserved[3] = 1
    t = mf.Tiles(A, opts)
    n = A.n
    b = torch.tensor(A.b(), device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    if args.kernel == "spmv":
        xs = torch.tensor(A.xstar() if A.xstar() is not None else np.ones(n), device="cuda")
        if args.time:
            ms, nbytes = t.spmv_bench(xs.data_ptr(), x.data_ptr(), args.reps, level)
            inf = t.info()
            print(f"spmv slab_bytes={args.slab_bytes} rb_per_slab={args.rb_per_slab} ctas={inf['nctas']} "
                  f"slabs={inf['nslabs']} ms={ms:.4f} GB/s={nbytes / ms / 1e6:.0f}")
            return
        for _ in range(args.reps):
            if level >= 0:
                t.spmv_level_dev(level, xs.data_ptr(), x.data_ptr())
            else:
                t.spmv_dev(xs.data_ptr(), x.data_ptr())
        torch.cuda.synchronize()
        print("spmv done", float(x.abs().sum()))
        return
    o = mf.options(fixed_iterations=args.iters, **kw)
    if args.trace > 0:
        o.reserved[1] = args.trace
    if args.prefetch:
        o.reserved[3] = 1
    if args.no_tmem:
        o.reserved[5] = 1
    if args.kernel in ("cg", "pcg"):
        fn = t.solve_cg_dev if args.kernel == "cg" else t.solve_pcg_dev
        res = fn(b.data_ptr(), x.data_ptr(), 1e-10, 40000, o)
        if args.trace > 0:
            tr = t.trace(args.trace).astype(np.float64)
            tr = tr[(tr[:, 0] > 0) & (tr[:, 6] > 0)]
            names = ["halo wait", "SpMV", "dot d.q", "r update", "dot r.r", "x/d update+publish"]
            if args.mode != "fp64":  # single-reduction CG
                names = ["halo wait", "SpMV (w = A r)", "reduction (r.r, w.r)", "p,s,x,r update", "-", "publish"]
            d = np.diff(tr[:, :7], axis=1) / 1e3
            it_us = np.diff(tr[:, 0]) / 1e3
            print("trace over %d iterations (us, median):" % len(tr))
            for k, nm in enumerate(names):
                print("  %-22s %8.2f" % (nm, np.median(d[:, k])))
            print("  %-22s %8.2f" % ("iteration", np.median(it_us)))
    else:
        res = t.solve_bicgstab_dev(b.data_ptr(), x.data_ptr(), 1e-10, 10000, o)
    torch.cuda.synchronize()
    print(args.kernel, res)


if __name__ == "__main__":
    main()
