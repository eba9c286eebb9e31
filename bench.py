"""Benchmark of the tiled CG hot path on one node.

Workload (the configuration the headline metric is quoted on): 3D 7-point
variable-coefficient Poisson on a 128^3 grid (n = 2,097,152, nnz =
14,581,760), face coefficients log-uniform in [1e-3, 1e3] (seed 1),
b = A x* with x* ~ U[0,1], x0 = 0, CG to a 1e-10 true relative residual.
One step = one complete solve. The matrix (172 MB in the FP64 tile format)
is larger than the 126 MB L2, so every SpMV streams from HBM; L2 is not
flushed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--mode fp64|mixed]
  python bench.py --impl reference ...   (CPU arm, see below)

N > 1 runs under torchrun, one rank per GPU: a single system does not
shard (every iteration needs grid-wide dot products), so each rank solves
its own replica (weak scaling, replicas only); the time is the max over
ranks. The reference arm times the CPU implementation of the same solve
(the oracle's restatement of the reference recurrence with the reference's
tiled SpMV order, OpenMP over all host cores) on a bounded sample of
iterations and projects the full solve by the iteration count.
"""
import argparse
import ctypes as C
import importlib
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solve time to 1e-10 true residual & SpMV HBM GB/s: mixed vs FP64, same B200"
N_GRID = 128
TOL = 1e-10
MAXITER = 40000
# Iterations of the FP64 recurrence to 1e-10 on this matrix, used to project
# the CPU arm's sampled per-iteration time to a full solve. Measured by the
# GPU FP64 solve, whose count the tests hold within 2 % of the CPU oracle.
FP64_ITERS_128 = None


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = os.path.join(ROOT, "gpurun_out", f"clocks_rank{device}.csv")

    def start(self):
        os.makedirs(os.path.dirname(self.path), exist_ok=True)
        try:
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.fh,
                                         stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        top = max(sm)
        loaded = [s for s in sm if s >= 0.5 * top] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def _dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        if args.impl == "reference":
            return world, rank, local, None
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        return world, rank, local, dist
    return world, rank, local, None


def _max_over_ranks(dist, value):
    if dist is None:
        return value
    import torch

    t = torch.tensor([value], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(dist):
    if dist is not None:
        dist.barrier()


def cpu_reference_arm(args, rank):
    """CPU CG of the reference recurrence (oracle port) on all host cores."""
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    mf = importlib.import_module("mille-feillue_b200")
    import _oracle as O

    A = mf.Matrix.varpoisson3d(N_GRID)
    n = A.n
    rp, ci, v = A.csr()
    b = A.b()
    t0 = time.perf_counter()
    o = O.OracleTiles(n, n, rp, ci, v)
    enc_s = time.perf_counter() - t0
    sample_iters = args.cpu_sample_iters
    times = []
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        it, _, _ = o.cg(b, 0.0, sample_iters)  # tol 0: exactly sample_iters iterations
        dt = time.perf_counter() - t0
        if step >= args.warmup:
            times.append(dt / max(it, 1))
    per_it = statistics.median(times)
    iters = args.fp64_iters or FP64_ITERS_128 or 0
    value = per_it * iters * 1e3 if iters else None
    cores = os.cpu_count()
    return {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "ms", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "varpoisson3d_128 CG to 1e-10 true residual", "n": n, "nnz": int(len(v)),
                   "x0": "zeros", "tol": TOL},
        "cpu_baseline": {"value": value, "unit": "ms", "cores": cores, "kind": "port",
                         "sample": f"{sample_iters} CG iterations of the oracle (reference recurrence, tiled "
                                   f"SpMV order, OpenMP) on the full matrix per step, median per-iteration "
                                   f"time x {iters} iterations to 1e-10", "ms_per_iteration": per_it * 1e3,
                         "tile_encode_s": enc_s},
        "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def gpu_arm(args, world, rank, local, dist):
    import torch

    mf = importlib.import_module("mille-feillue_b200")
    dev = local
    torch.cuda.set_device(dev)
    A = mf.Matrix.varpoisson3d(N_GRID)
    n = A.n
    rp, ci, v = A.csr()
    b = A.b()
    xstar = A.xstar()
    mode = args.mode
    popts = dict(device=dev)
    if mode == "mixed":
        popts.update(precision_mode=mf.MODE_MIXED_RULE)
    opts = mf.options(**popts)
    t_enc0 = time.perf_counter()
    tiles = mf.Tiles(A, opts)
    enc_s = time.perf_counter() - t_enc0
    info = tiles.info()
    bd = torch.tensor(b, device=f"cuda:{dev}")
    xd = torch.zeros(n, dtype=torch.float64, device=f"cuda:{dev}")
    launches_per_solve = 3  # persistent solver kernel + true-residual SpMV + norm kernel

    # ---- standalone SpMV (FP64 layout): roofline of the streamed kernel
    xs = torch.tensor(xstar, device=f"cuda:{dev}")
    ys = torch.zeros(n, dtype=torch.float64, device=f"cuda:{dev}")
    spmv_ms, spmv_bytes = tiles.spmv_bench(xs.data_ptr(), ys.data_ptr(), 50)
    peak, peak_kind = _peaks()

    # ---- warm-up solves
    for _ in range(args.warmup):
        xd.zero_()
        res = tiles.solve_cg_dev(bd.data_ptr(), xd.data_ptr(), TOL, MAXITER, opts)
    torch.cuda.synchronize()
    _barrier(dist)
    clocks = ClockSampler(dev)
    clocks.start()
    torch.cuda.synchronize()
    _barrier(dist)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    kernel_ms = []
    e0.record()
    for _ in range(args.steps):
        xd.zero_()
        res = tiles.solve_cg_dev(bd.data_ptr(), xd.data_ptr(), TOL, MAXITER, opts)
        kernel_ms.append(res["time_ms"])
    e1.record()
    torch.cuda.synchronize()
    _barrier(dist)
    ms = e0.elapsed_time(e1) / args.steps
    ms = _max_over_ranks(dist, ms)
    clk = clocks.stop()
    x = xd.cpu().numpy()
    err = float(np.linalg.norm(x - xstar) / np.linalg.norm(xstar))

    # ---- end to end through the C ABI with pinned host buffers:
    # CSR + b host->device, GPU encode, persistent solve, x device->host
    rp_h = torch.from_numpy(rp).pin_memory()
    ci_h = torch.from_numpy(ci).pin_memory()
    v_h = torch.from_numpy(v).pin_memory()
    b_h = torch.from_numpy(b).pin_memory()
    x_h = torch.zeros(n, dtype=torch.float64).pin_memory()
    L = mf.lib()
    csr = mf.MfCsr(n, n, int(len(v)), rp_h.data_ptr(), ci_h.data_ptr(), v_h.data_ptr())
    e2e = []
    for step in range(1 + max(1, args.e2e_steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h = mf._p()
        rc = L.mf_encode(C.byref(csr), C.byref(opts), C.byref(h))
        assert rc == 0, rc
        x_h.zero_()
        r2 = mf.MfResult()
        rc = L.mf_solve_cg(h, C.c_void_p(b_h.data_ptr()), C.c_void_p(x_h.data_ptr()), TOL, MAXITER,
                           C.byref(opts), C.byref(r2))
        L.mf_free(h)
        torch.cuda.synchronize()
        if step > 0:
            e2e.append((time.perf_counter() - t0) * 1e3)
    e2e_ms = _max_over_ranks(dist, statistics.median(e2e))
    h2d = rp.nbytes + ci.nbytes + v.nbytes + b.nbytes + n * 8  # CSR, b, x0
    d2h = n * 8 + 8  # x and the result scalars

    iters = res["iterations"]
    it_bytes = spmv_bytes + 56.0 * n  # per-iteration algorithmic bytes (SpMV + fused vector pass)
    solve_gbs = iters * it_bytes / (statistics.median(kernel_ms) * 1e-3) / 1e9
    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "varpoisson3d_128 CG to 1e-10 true residual", "n": n, "nnz": int(len(v)),
                       "mode": mode, "x0": "zeros", "tol": TOL, "parallelism": "replicas" if world > 1 else "single",
                       "l2": "matrix (%.0f MB) larger than L2; not flushed" % (spmv_bytes / 1e6),
                       "ctas": info["nctas"], "slabs": info["nslabs"]},
            "iterations": iters, "rel_residual_true": res["rel_residual_true"], "x_err_vs_xstar": err,
            "kernel_ms": statistics.median(kernel_ms),
            "roofline": {"bound": "hbm", "achieved": solve_gbs, "peak": peak, "unit": "GB/s",
                         "frac": solve_gbs / peak, "traffic": None, "peak_kind": peak_kind,
                         "kernel": "k_cg (persistent solve), bytes = iterations x (B_spmv + 56 n)"},
            "spmv": {"ms": spmv_ms, "alg_bytes": spmv_bytes, "gbs": spmv_bytes / spmv_ms / 1e6,
                     "frac": spmv_bytes / spmv_ms / 1e6 / peak,
                     "gflops": 2.0 * len(v) / spmv_ms / 1e6},
            "clocks": clk,
            "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "path": "mf_encode(host CSR) + mf_solve_cg(host b, host x) + mf_free"},
            "gpu_launches": args.steps * launches_per_solve,
            "encode_s": enc_s, "encode_ms_device": info["encode_ms"], "layout_ms": info["layout_ms"],
        }
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--cpu-sample-iters", type=int, default=20)
    ap.add_argument("--fp64-iters", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    world, rank, local, dist = _dist_setup(args)
    if args.impl == "reference":
        out = cpu_reference_arm(args, rank)
        if out is not None:
            print(json.dumps(out))
        return
    out = gpu_arm(args, world, rank, local, dist)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        a2 = argparse.Namespace(**vars(args))
        a2.steps, a2.warmup = 1, 1
        a2.fp64_iters = args.fp64_iters or out["iterations"] if args.mode == "fp64" else args.fp64_iters
        ref = cpu_reference_arm(a2, 0)
        out["cpu_baseline"] = ref["cpu_baseline"]
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
