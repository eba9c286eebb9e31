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
tiled SpMV order, OpenMP over all host cores): one whole solve to the
tolerance per step, on a matrix built by the oracle's own generator (the
product library is not loaded in that arm).
"""
import argparse
import ctypes as C
import importlib
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solve time to 1e-10 true residual & SpMV HBM GB/s: mixed vs FP64, same B200"
N_GRID = 128
TOL = 1e-10
MAXITER = 40000


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
        self.path = os.path.join(tempfile.gettempdir(), f"mf_bench_clocks_rank{device}.csv")

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

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def _barrier(dist):
    if dist is not None:
        dist.barrier()


def _cpu_spmv_reference(O, n, rp, ci, v, x):
    """The reference's own blockspmv_cpu (compiled unmodified from its
    sources into oracle/_ref) on the same matrix: serial as in the reference
    (1 core), best of 10 after 2 warm-ups; its own Tile_create (OpenMP) is
    timed apart."""
    if not os.path.exists(O.REF_SO):
        return {"unavailable": "oracle/_ref/libmfref.so not built (needs the reference sources at build time)"}
    t0 = time.perf_counter()
    R = O.RefTiles(n, n, rp, ci, v)
    create_s = time.perf_counter() - t0
    times = []
    for rep in range(12):
        t0 = time.perf_counter()
        R.spmv(x)
        if rep >= 2:
            times.append(time.perf_counter() - t0)
    ms = min(times) * 1e3
    sz = R.sizes
    alg = 9.0 * sz["csrsize"] + 8.0 * sz["tilenum"] + 16.0 * n  # FP64 values + 1-byte columns, tile index, x, y
    return {"kind": "reference", "cores": 1, "ms": ms, "alg_bytes": alg, "gbs": alg / ms / 1e6,
            "tile_create_s": create_s,
            "sample": "blockspmv_cpu of the reference (serial, as shipped) on the full matrix, FP64; best of 10 "
                      "after 2 warm-ups, each call with the reference's own per-call allocations"}


def _cpu_small_configs(O):
    """Full oracle solves (all host cores, best of 3) of the two smaller
    configurations: C1 = CG on the 2D 5-point Poisson 256^2, C2 = BiCGSTAB
    on the 3D convection-diffusion 64^3, both to 1e-10 from x0 = 0."""
    out = {}
    for name, S, solver in (("C1_poisson2d_256_cg", O.gen_poisson2d(256), "cg"),
                            ("C2_convdiff3d_64_bicgstab", O.gen_convdiff3d(64), "bicgstab")):
        o = O.OracleTiles(S.n, S.n, *S.csr())
        best, it, rel = None, 0, 0.0
        for _ in range(3):
            t0 = time.perf_counter()
            it, _, rel = getattr(o, solver)(S.b, TOL, MAXITER)
            dt = (time.perf_counter() - t0) * 1e3
            best = dt if best is None else min(best, dt)
        out[name] = {"ms": best, "iterations": int(it), "rel_residual": float(rel)}
    return out


def _config(world, grid):
    """The workload of both arms (identical keys and values). The 7-point
    matrix of a grid^3 problem has 7 n - 6 grid^2 nonzeros."""
    l2 = ("matrix (172 MB in the FP64 tile format) larger than the 126 MB L2; not flushed" if grid == 128
          else "reduced grid (test size): the matrix may sit in L2; not flushed")
    return {"workload": f"varpoisson3d_{grid} CG to 1e-10 true residual", "n": grid ** 3,
            "nnz": 7 * grid ** 3 - 6 * grid ** 2, "x0": "zeros", "tol": TOL,
            "parallelism": "replicas" if world > 1 else "single", "l2": l2}


def cpu_reference_arm(args, rank, world=1, small=True):
    """CPU CG of the reference recurrence (the oracle's restatement, tiled
    SpMV in the reference's order, OpenMP over all host cores): every step is
    one whole solve of the headline system to the tolerance, timed on its
    own. The matrix comes from the oracle's generator; the product library
    is not loaded. Beside it, the reference's own serial blockspmv_cpu."""
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import _oracle as O

    # every host core this process may run on (torchrun sets OMP_NUM_THREADS=1)
    cores = O.set_threads(len(os.sched_getaffinity(0)))

    S = O.gen_varpoisson3d(args.grid)
    n = S.n
    rp, ci, v = S.csr()
    t0 = time.perf_counter()
    o = O.OracleTiles(n, n, rp, ci, v)
    enc_s = time.perf_counter() - t0
    times, iters, rel, err = [], 0, 0.0, None
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        iters, x, rel = o.cg(S.b, TOL, MAXITER)
        dt = (time.perf_counter() - t0) * 1e3
        if step >= args.warmup:
            times.append(dt)
            err = float(np.linalg.norm(x - S.xstar) / np.linalg.norm(S.xstar))
    value = statistics.median(times)
    try:
        spmv_ref = _cpu_spmv_reference(O, n, rp, ci, v, S.xstar)
    except (OSError, RuntimeError, ValueError) as e:  # the solve's baseline stands without it
        spmv_ref = {"unavailable": f"{type(e).__name__}: {e}"}
    out = {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "ms", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": value, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _config(world, args.grid), "mode": "fp64",
        "cpu_baseline": {"value": value, "unit": "ms", "cores": cores, "kind": "port",
                         "sample": f"one whole FP64 CG solve to 1e-10 per step ({int(iters)} iterations of the "
                                   f"oracle: reference recurrence, tiled SpMV in the reference's order, OpenMP on "
                                   f"{cores} threads), median of {args.steps} steps after {args.warmup} warm-up "
                                   f"solves; matrix from the oracle's generator",
                         "iterations": int(iters), "rel_residual": float(rel), "x_err_vs_xstar": err,
                         "step_ms_min_max": [min(times), max(times)], "tile_encode_s": enc_s,
                         "spmv_reference_1core": spmv_ref},
        "e2e": {"value": value, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    if small:
        out["cpu_baseline"]["other_configs"] = _cpu_small_configs(O)
    return out


def _time_solves(torch, tiles, bd, xd, opts, steps, warmup, dist, solver="cg"):
    res = None
    solve = tiles.solve_pcg_dev if solver == "pcg" else tiles.solve_cg_dev
    for _ in range(warmup):
        xd.zero_()
        res = solve(bd.data_ptr(), xd.data_ptr(), TOL, MAXITER, opts)
    torch.cuda.synchronize()
    _barrier(dist)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    kernel_ms = []
    e0.record()
    for _ in range(steps):
        xd.zero_()
        res = solve(bd.data_ptr(), xd.data_ptr(), TOL, MAXITER, opts)
        kernel_ms.append(res["time_ms"])
    e1.record()
    torch.cuda.synchronize()
    _barrier(dist)
    ms = _max_over_ranks(dist, e0.elapsed_time(e1) / steps)
    return ms, statistics.median(kernel_ms), res


def gpu_arm(args, world, rank, local, dist):
    import torch

    mf = importlib.import_module("mille-feillue_b200")
    dev = local
    torch.cuda.set_device(dev)
    A = mf.Matrix.varpoisson3d(args.grid)
    n = A.n
    rp, ci, v = A.csr()
    b = A.b()
    xstar = A.xstar()
    opts64 = mf.options(device=dev)
    optsmx = mf.options(device=dev, precision_mode=mf.MODE_MIXED_RULE)
    t_enc0 = time.perf_counter()
    tiles = mf.Tiles(A, optsmx)  # FP64 layout + mixed-precision levels
    enc_s = time.perf_counter() - t_enc0
    info = tiles.info()
    bd = torch.tensor(b, device=f"cuda:{dev}")
    xd = torch.zeros(n, dtype=torch.float64, device=f"cuda:{dev}")
    launches_per_solve = 3  # persistent solver kernel + true-residual SpMV + norm kernel
    headline = args.mode
    opts = optsmx if headline == "mixed" else opts64

    # ---- standalone SpMV: roofline of the streamed kernel (FP64 and level 0)
    xs = torch.tensor(xstar, device=f"cuda:{dev}")
    ys = torch.zeros(n, dtype=torch.float64, device=f"cuda:{dev}")
    spmv_ms, spmv_bytes = tiles.spmv_bench(xs.data_ptr(), ys.data_ptr(), 50)
    spmv_mx_ms, spmv_mx_bytes = tiles.spmv_bench(xs.data_ptr(), ys.data_ptr(), 50, level=0)
    peak, peak_kind = _peaks()

    clocks = ClockSampler(dev)
    clocks.start()
    ms64, k64, res64 = _time_solves(torch, tiles, bd, xd, opts64, args.steps, args.warmup, dist)
    x64 = xd.cpu().numpy()
    msmx, kmx, resmx = _time_solves(torch, tiles, bd, xd, optsmx, args.steps, args.warmup, dist)
    xmx = xd.cpu().numpy()
    clk = clocks.stop()
    # Jacobi-preconditioned CG (FP64), reported beside the headline
    mspc, kpc, respc = _time_solves(torch, tiles, bd, xd, opts64, max(1, args.steps // 2), 1, dist, "pcg")
    errpc = float(np.linalg.norm(xd.cpu().numpy() - xstar) / np.linalg.norm(xstar))
    # the same FP64 CG built from cuSPARSE + cuBLAS calls (baseline/cusparse)
    vs_cusp = None
    Lc = _cusp_lib() if rank == 0 and not args.no_cusparse else None
    if Lc is not None:
        _cusp_solve(Lc, "cg", A, b, 0.0, 5)
        cu = _cusp_solve(Lc, "cg", A, b, TOL, MAXITER)
        vs_cusp = {"cusparse_cg_fp64_ms": cu["ms"], "cusparse_iterations": cu["iterations"],
                   "ours_fp64_ms": ms64, "ours_mixed_ms": msmx, "speedup_fp64": cu["ms"] / ms64,
                   "speedup_mixed": cu["ms"] / msmx,
                   "baseline": "cuSPARSE CSR SpMV (ALG_DEFAULT) + cuBLAS level 1, host-side scalars"}
    nx = np.linalg.norm(x64)
    err64 = float(np.linalg.norm(x64 - xstar) / np.linalg.norm(xstar))
    errmx = float(np.linalg.norm(xmx - xstar) / np.linalg.norm(xstar))
    mx_vs_64 = float(np.linalg.norm(xmx - x64) / nx)
    ms, kms, res = (msmx, kmx, resmx) if headline == "mixed" else (ms64, k64, res64)
    if headline == "mixed":
        names = ("FP64", "FP32", "FP16", "FP8-E4M3")
        used = [f"{names[i]} {100 * f:.0f}%" for i, f in enumerate(resmx["tile_frac"]) if f > 0]
        dtype = "mixed: tile values " + ", ".join(used) + "; FP64 vectors, dots, scalars"
    else:
        dtype = "f64"

    # ---- end to end through the C ABI with pinned host buffers:
    # CSR + b host->device, GPU encode, persistent solve, x device->host
    rp_h = torch.from_numpy(rp).pin_memory()
    ci_h = torch.from_numpy(ci).pin_memory()
    v_h = torch.from_numpy(v).pin_memory()
    b_h = torch.from_numpy(b).pin_memory()
    x_h = torch.zeros(n, dtype=torch.float64).pin_memory()
    L = mf.lib()
    csr = mf.MfCsr(n, n, int(len(v)), rp_h.data_ptr(), ci_h.data_ptr(), v_h.data_ptr())
    e2e, parts = [], []
    for step in range(1 + max(1, args.e2e_steps)):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        h = mf._p()
        rc = L.mf_encode(C.byref(csr), C.byref(opts), C.byref(h))
        assert rc == 0, rc
        t1 = time.perf_counter()
        x_h.zero_()
        r2 = mf.MfResult()
        rc = L.mf_solve_cg(h, C.c_void_p(b_h.data_ptr()), C.c_void_p(x_h.data_ptr()), TOL, MAXITER,
                           C.byref(opts), C.byref(r2))
        t2 = time.perf_counter()
        L.mf_free(h)
        torch.cuda.synchronize()
        t3 = time.perf_counter()
        if step > 0:
            e2e.append((t3 - t0) * 1e3)
            parts.append(((t1 - t0) * 1e3, (t2 - t1) * 1e3, (t3 - t2) * 1e3))
    e2e_ms = _max_over_ranks(dist, statistics.median(e2e))
    e2e_parts = {k: statistics.median(p[i] for p in parts) for i, k in enumerate(("encode_ms", "solve_ms", "free_ms"))}
    h2d = rp.nbytes + ci.nbytes + v.nbytes + b.nbytes + n * 8  # CSR, b, x0
    d2h = n * 8 + 8  # x and the result scalars

    def roof(r, kernel_ms):
        gbs = r["total_bytes"] / (kernel_ms * 1e-3) / 1e9
        return gbs

    gbs = roof(res, kms)
    # DRAM bytes per CG iteration (read + write) measured with ncu as the
    # difference of a 40- and a 20-iteration launch of the same matrix
    # (dram__bytes_read + write; profiles/k_cg_tm_k_cgcg_tm_varpoisson128.md),
    # scaled by the iterations of the timed solve (plus the initial and the
    # replacement FP64 SpMVs at their algorithmic bytes)
    dram_per_iter = {"mixed": 44.2e6, "fp64": 150.4e6}[headline]
    traffic = res["iterations"] * dram_per_iter + (1 + res["replacements"]) * spmv_bytes
    kname = ("k_cgcg_tm (mixed single-reduction CG, x and r in tensor memory)" if headline == "mixed"
             else "k_cg_tm (FP64 CG, x and r in tensor memory)")
    out = None
    if rank == 0:
        out = {
            "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": dtype, "data": "synthetic",
            "config": _config(world, args.grid), "mode": headline,
            "layout": {"ctas": info["nctas"], "slabs": info["nslabs"], "spmv_fp64_alg_bytes": spmv_bytes},
            "iterations": res["iterations"], "rel_residual_true": res["rel_residual_true"],
            "mixed": {"ms": msmx, "kernel_ms": kmx, "iterations": resmx["iterations"],
                      "iters_per_level": resmx["iters_level"], "replacements": resmx["replacements"],
                      "level_switches": resmx["level_switches"], "tile_frac_final": resmx["tile_frac"],
                      "rel_residual_true": resmx["rel_residual_true"], "x_err_vs_xstar": errmx,
                      "x_diff_vs_fp64": mx_vs_64, "spmv_bytes_level": resmx["spmv_bytes_level"]},
            "fp64": {"ms": ms64, "kernel_ms": k64, "iterations": res64["iterations"],
                     "rel_residual_true": res64["rel_residual_true"], "x_err_vs_xstar": err64,
                     "roofline_gbs": roof(res64, k64), "roofline_frac": roof(res64, k64) / peak},
            "speedup_mixed_vs_fp64": ms64 / msmx,
            "vs_cusparse": vs_cusp,
            "fp64_jacobi_pcg": {"ms": mspc, "kernel_ms": kpc, "iterations": respc["iterations"],
                                "rel_residual_true": respc["rel_residual_true"], "x_err_vs_xstar": errpc,
                                "speedup_vs_fp64_cg": ms64 / mspc},
            "roofline": {"bound": "hbm", "achieved": gbs, "peak": peak, "unit": "GB/s", "frac": gbs / peak,
                         "traffic": traffic, "peak_kind": peak_kind,
                         "kernel": kname + "; one launch = one solve; algorithmic bytes = every SpMV's "
                                   "algorithmic bytes + the vector bytes the kernel moves per iteration "
                                   "(28 n mixed, 32 n FP64: x and r stay in tensor memory)",
                         "dram_bytes_per_iteration_measured": dram_per_iter},
            "spmv": {"fp64": {"ms": spmv_ms, "alg_bytes": spmv_bytes, "gbs": spmv_bytes / spmv_ms / 1e6,
                              "frac": spmv_bytes / spmv_ms / 1e6 / peak, "gflops": 2.0 * len(v) / spmv_ms / 1e6},
                     "mixed_level0": {"ms": spmv_mx_ms, "alg_bytes": spmv_mx_bytes,
                                      "gbs": spmv_mx_bytes / spmv_mx_ms / 1e6,
                                      "frac": spmv_mx_bytes / spmv_mx_ms / 1e6 / peak,
                                      "gflops": 2.0 * len(v) / spmv_mx_ms / 1e6}},
            "clocks": clk,
            "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    **e2e_parts,
                    "path": "mf_encode(host CSR) + mf_solve_cg(host b, host x) + mf_free"},
            "gpu_launches": args.steps * launches_per_solve,
            "encode_s": enc_s, "encode_ms_device": info["encode_ms"], "layout_ms": info["layout_ms"],
        }
    return out


def _cusp_lib():
    """The cuSPARSE + cuBLAS CG / BiCGSTAB of baseline/cusparse (built by
    __graft_entry__.build())."""
    path = os.path.join(ROOT, "baseline", "cusparse", "libcusp.so")
    if not os.path.exists(path):
        return None
    L = C.CDLL(path)
    for f in ("cusp_cg", "cusp_bicgstab"):
        getattr(L, f).argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_double, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                  C.POINTER(C.c_double)]
    return L


def _cusp_solve(L, solver, A, b, tol, maxiter):
    rp, ci, v = A.csr()
    rp = np.ascontiguousarray(rp, np.int32)
    ci = np.ascontiguousarray(ci, np.int32)
    v = np.ascontiguousarray(v, np.float64)
    b = np.ascontiguousarray(b, np.float64)
    x = np.zeros(A.n)
    it, ms, rel = C.c_int(), C.c_double(), C.c_double()
    fn = L.cusp_cg if solver == "cg" else L.cusp_bicgstab
    rc = fn(A.n, len(v), rp.ctypes.data, ci.ctypes.data, v.ctypes.data, b.ctypes.data, x.ctypes.data, tol, maxiter,
            C.byref(it), C.byref(ms), C.byref(rel))
    assert rc == 0, rc
    return {"ms": ms.value, "iterations": it.value, "rel_residual": rel.value}


def _ours_solve(torch, mf, A, b, solver, tol, fixed, dev, reps=3):
    t = mf.Tiles(A, mf.options(device=dev))
    bd = torch.tensor(b, device=f"cuda:{dev}")
    xd = torch.zeros(A.n, dtype=torch.float64, device=f"cuda:{dev}")
    o = mf.options(device=dev, fixed_iterations=fixed)
    fn = t.solve_cg_dev if solver == "cg" else t.solve_bicgstab_dev
    best = None
    for _ in range(reps):
        xd.zero_()
        r = fn(bd.data_ptr(), xd.data_ptr(), tol, MAXITER, o)
        if best is None or r["time_ms"] < best["time_ms"]:
            best = r
    return {"ms": best["time_ms"], "iterations": best["iterations"], "rel_residual": best["rel_residual_true"]}


def cusparse_arm(args, rank, local):
    """FP64 CG / BiCGSTAB of libmf against cuSPARSE + cuBLAS loops on the
    same GPU: C1 (CG, 2D Poisson 256^2), C2 (BiCGSTAB, 3D convection-diffusion
    64^3), C3 (CG, 128^3 variable-coefficient Poisson); to 1e-10 and for a
    fixed 100 iterations (the reference's own comparison runs 100)."""
    if rank != 0:
        return None
    import torch

    mf = importlib.import_module("mille-feillue_b200")
    torch.cuda.set_device(local)
    L = _cusp_lib()
    if L is None:
        return {"metric": "speedup over cuSPARSE CG / BiCGSTAB", "unavailable": "baseline/cusparse not built"}
    cases = [("C1_poisson2d_256_cg", mf.Matrix.poisson2d(256), "cg"),
             ("C2_convdiff3d_64_bicgstab", mf.Matrix.convdiff3d(64), "bicgstab"),
             ("C3_varpoisson3d_128_cg", mf.Matrix.varpoisson3d(N_GRID), "cg")]
    rows = {}
    for name, A, solver in cases:
        b = A.b()
        _cusp_solve(L, solver, A, b, 0.0, 5)  # warm
        cu = min((_cusp_solve(L, solver, A, b, TOL, MAXITER) for _ in range(2)), key=lambda r: r["ms"])
        cu100 = min((_cusp_solve(L, solver, A, b, 0.0, 100) for _ in range(2)), key=lambda r: r["ms"])
        ours = _ours_solve(torch, mf, A, b, solver, TOL, 0, local)
        ours100 = _ours_solve(torch, mf, A, b, solver, TOL, 100, local)
        rows[name] = {"cusparse": cu, "ours_fp64": ours,
                      "speedup_to_tol": cu["ms"] / ours["ms"],
                      "cusparse_us_per_iteration_100": cu100["ms"] * 10.0,
                      "ours_us_per_iteration_100": ours100["ms"] * 10.0,
                      "speedup_per_iteration_100": cu100["ms"] / ours100["ms"]}
    sp = [r["speedup_to_tol"] for r in rows.values()]
    return {"metric": "speedup over cuSPARSE CG / BiCGSTAB (time to 1e-10, FP64, same B200)",
            "value": float(np.exp(np.mean(np.log(sp)))), "unit": "x (geomean)", "n_gpus": 1,
            "higher_is_better": True, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "C1 CG, C2 BiCGSTAB, C3 CG; cuSPARSE CSR SpMV (ALG_DEFAULT) + cuBLAS level 1, "
                                   "host-side scalars, x0 = 0"},
            "cases": rows}


def multi_rhs_arm(args, rank, local, fp64_panel=False):
    """CG on 16 right-hand sides at once (one shared panel product per
    iteration; FP32 search directions and products, FP64 x, r, dots and
    scalars, one persistent launch) against 16 single-right-hand-side FP64
    solves of the same columns (the tensor-memory CG kernel), on the 128^3
    variable-coefficient Poisson matrix with 16 seeded U[-1, 1] right-hand
    sides; device time of each solve to a 1e-10 relative residual (the true
    one for the panel solve). fp64_panel adds the exact FP64-panel path."""
    if rank != 0:
        return None
    import torch

    mf = importlib.import_module("mille-feillue_b200")
    torch.cuda.set_device(local)
    A = mf.Matrix.varpoisson3d(N_GRID)
    n = A.n
    B = np.random.default_rng(7).uniform(-1, 1, (n, 16))
    mf.solve_cg_multi(A, B[:, :2], tol=TOL, maxiter=50)  # warm
    X, it, rel, multi_ms = mf.solve_cg_multi(A, B, tol=TOL, maxiter=MAXITER)
    t = mf.Tiles(A)
    x = torch.zeros(n, dtype=torch.float64, device=f"cuda:{local}")
    b0 = torch.tensor(np.ascontiguousarray(B[:, 0]), device=f"cuda:{local}")
    t.solve_cg_dev(b0.data_ptr(), x.data_ptr(), TOL, 50)  # warm
    single_ms, single_it, xdiff = 0.0, [], 0.0
    for j in range(16):
        b = torch.tensor(np.ascontiguousarray(B[:, j]), device=f"cuda:{local}")
        x.zero_()
        r = t.solve_cg_dev(b.data_ptr(), x.data_ptr(), TOL, MAXITER)
        single_ms += r["time_ms"]
        single_it.append(int(r["iterations"]))
        xs = x.cpu().numpy()
        xdiff = max(xdiff, float(np.linalg.norm(X[:, j] - xs) / np.linalg.norm(xs)))
    out = {"metric": "16-RHS CG time to 1e-10 (shared panel product) vs 16 single-RHS solves",
           "value": multi_ms, "unit": "ms", "n_gpus": 1, "higher_is_better": False,
           "dtype": "FP32 search directions and panel products; FP64 x, r, dots, scalars",
           "data": "synthetic",
           "config": {"workload": "varpoisson3d 128^3, 16 RHS U[-1,1] seed 7, x0 = 0, CG to 1e-10 per column"},
           "iterations_min_max": [int(it.min()), int(it.max())], "max_rel_residual": float(rel.max()),
           "single_rhs_total_ms": single_ms, "single_iterations_min_max": [min(single_it), max(single_it)],
           "max_x_diff_vs_single": xdiff, "speedup_vs_single_rhs": single_ms / multi_ms}
    if fp64_panel:
        _, it64, rel64, ms64 = mf.solve_cg_multi(A, B, tol=TOL, maxiter=MAXITER, panel=mf.PANEL_FP64)
        out["fp64_panel"] = {"ms": ms64, "iterations_min_max": [int(it64.min()), int(it64.max())],
                             "max_rel_residual": float(rel64.max()), "speedup_vs_single_rhs": single_ms / ms64}
    return out


def batch_arm(args, world, rank, local, dist, steps=None, warmup=None):
    """512 random SPD systems, n log-uniform in [1e3, 2e5] (seed 2), FP64 CG
    to 1e-10: one persistent launch (CUDA-graph replay) against one
    single-system launch per system. With N ranks the systems are split by
    longest-processing-time on nnz (no collective in the solve)."""
    import torch

    mf = importlib.import_module("mille-feillue_b200")
    dev = local
    torch.cuda.set_device(dev)
    sizes = mf.batch_sizes(512, 1000, 200000, 2)
    # LPT split of the systems over ranks by size (nnz grows with n)
    mine = mf.split_systems(sizes, world)[rank]
    t0 = time.perf_counter()
    mats = mf.generate_spd_batch([sizes[s] for s in mine], seed=2, index=mine)
    gen_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    bopt = mf.options(device=dev)
    bopt.reserved[4] = args.batch_group  # CTAs per system group (0 = library default)
    B = mf.Batch(mats, bopt, with_baseline=not args.no_each)
    enc_s = time.perf_counter() - t0
    b = np.concatenate([m.b() for m in mats])
    bd = torch.tensor(b, device=f"cuda:{dev}")
    xd = torch.zeros_like(bd)
    steps = args.steps if steps is None else steps
    warmup = args.warmup if warmup is None else warmup
    for _ in range(warmup):
        B.solve_cg_dev(bd.data_ptr(), xd.data_ptr(), TOL, 10000)
    torch.cuda.synchronize()
    _barrier(dist)
    clocks = ClockSampler(dev)
    clocks.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        B.solve_cg_dev(bd.data_ptr(), xd.data_ptr(), TOL, 10000)
    e1.record()
    torch.cuda.synchronize()
    _barrier(dist)
    clk = clocks.stop()
    ms = _max_over_ranks(dist, e0.elapsed_time(e1) / steps)
    it, st, rel = B.results()
    each_ms = None
    if not args.no_each:
        xe = torch.zeros_like(bd)
        B.solve_cg_each_dev(bd.data_ptr(), xe.data_ptr(), TOL, 10000)  # warm
        each_ms = _max_over_ranks(dist, B.solve_cg_each_dev(bd.data_ptr(), xe.data_ptr(), TOL, 10000))
    inf = B.info()
    if rank != 0:
        return None
    return {
        "metric": "batched solve time to 1e-10 (512 SPD systems)", "value": ms, "unit": "ms", "n_gpus": world,
        "steps": steps, "warmup": warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": "batch512_spd n~logU[1e3,2e5] seed 2, CG to 1e-10", "systems": len(mats),
                   "rows_rank0": inf["rows"], "nnz_rank0": inf["nnz"], "grid": inf["grid"],
                   "ctas_per_group": args.batch_group or 4,
                   "parallelism": f"systems split over {world} ranks (LPT)" if world > 1 else "single"},
        "iterations_min_max": [int(it.min()), int(it.max())], "all_converged": bool(np.all(st == 0)),
        "max_rel_residual": float(rel.max()),
        "one_launch_per_system_ms": each_ms,
        "speedup_vs_one_launch_per_system": (each_ms / ms) if each_ms else None,
        "clocks": clk, "gen_s": gen_s, "encode_s": enc_s,
        "gpu_launches": steps * 3,
    }


def _extra_legs(args, world, rank, local, dist, out):
    """The two other workloads of the solver, measured in the default run
    beside the headline: the batched 512-system launch against one launch
    per system (systems split over the ranks), and CG on 16 right-hand sides
    against 16 single solves (rank 0 of a one-GPU run)."""
    if args.no_extra:
        return
    try:
        bat = batch_arm(args, world, rank, local, dist, steps=3, warmup=1)
    except Exception as e:  # the headline stands without it
        bat = {"unavailable": f"{type(e).__name__}: {e}"}
    if rank == 0 and out is not None:
        keep = ("value", "unit", "n_gpus", "steps", "warmup", "config", "iterations_min_max", "all_converged",
                "max_rel_residual", "one_launch_per_system_ms", "speedup_vs_one_launch_per_system", "clocks",
                "encode_s", "unavailable")
        out["batch512"] = {k: bat[k] for k in keep if bat and k in bat}
    if rank == 0 and world == 1 and out is not None:
        try:
            m = multi_rhs_arm(args, rank, local)
            out["multi16"] = {k: m[k] for k in ("value", "unit", "dtype", "config", "iterations_min_max",
                                                "max_rel_residual", "single_rhs_total_ms",
                                                "single_iterations_min_max", "max_x_diff_vs_single",
                                                "speedup_vs_single_rhs")}
        except Exception as e:
            out["multi16"] = {"unavailable": f"{type(e).__name__}: {e}"}


def profile_case(args):
    """One kernel of the solver on a fixed workload, for profilers
    (`--workload profile`):

      spmv      `--reps` launches of the tiled SpMV (k_spmv) on x*; with
                `--time`, the CUDA-event time of 50-launch batches instead
      cg / pcg  one persistent-solver launch of `--iters` iterations
                (0 = to the 1e-10 tolerance); `--trace N` prints the median
                phase times of the first N CG iterations
      bicgstab  the same on the convection-diffusion matrix
      multi     CG on 16 right-hand sides (U[-1, 1], seed 0), `--iters`
                iterations: the persistent FP32-panel kernel, or with
                `--prec fp64` the FP64 panel's product, scalar and update
                kernels

    Matrix: the 3D variable-coefficient Poisson (cg, pcg, spmv, multi) or
    convection-diffusion (bicgstab) of `--grid`. `--prec` picks the storage:
    fp64, mixed (the magnitude rule's first level), or all tiles fixed at
    fp32 / fp16 / fp8."""
    import torch

    mf = importlib.import_module("mille-feillue_b200")
    A = mf.Matrix.convdiff3d(args.grid) if args.kernel == "bicgstab" else mf.Matrix.varpoisson3d(args.grid)
    if args.kernel == "multi":
        B = np.random.default_rng(0).uniform(-1, 1, (A.n, 16))
        panel = mf.PANEL_FP64 if args.prec == "fp64" else mf.PANEL_FP32
        X, it, rel, ms = mf.solve_cg_multi(A, B, tol=1e-30, maxiter=args.iters, panel=panel)
        print("multi 16 rhs (%s panel): %d iterations %.2f ms -> %.1f us/iteration"
              % ("fp64" if panel == mf.PANEL_FP64 else "fp32", int(it.max()), ms, ms * 1e3 / max(1, int(it.max()))))
        return
    prec = args.prec or args.mode
    kw, level = {}, -1
    if prec == "mixed":
        kw, level = dict(precision_mode=mf.MODE_MIXED_RULE), 0
    elif prec in ("fp32", "fp16", "fp8"):
        kw = dict(precision_mode=mf.MODE_FIXED, fixed_precision={"fp32": 1, "fp16": 2, "fp8": 3}[prec])
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
        res = fn(b.data_ptr(), x.data_ptr(), 1e-10, MAXITER, o)
        if args.trace > 0:
            tr = t.trace(args.trace).astype(np.float64)
            tr = tr[(tr[:, 0] > 0) & (tr[:, 6] > 0)]
            names = ["halo wait", "SpMV", "dot d.q", "r update", "dot r.r", "x/d update+publish"]
            if prec != "fp64":  # single-reduction CG
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--mode", default="mixed", choices=["fp64", "mixed"])
    ap.add_argument("--grid", type=int, default=N_GRID,
                    help="grid edge of the headline Poisson system (128 = the measured configuration; "
                         "smaller only for quick checks)")
    ap.add_argument("--e2e-steps", type=int, default=5)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-cusparse", action="store_true", help="skip the cuSPARSE + cuBLAS comparison leg")
    ap.add_argument("--no-extra", action="store_true", help="skip the batch512 / multi16 legs of the default run")
    ap.add_argument("--workload", default="poisson128",
                    choices=["poisson128", "batch", "vs_cusparse", "multi16", "profile"])
    # --workload profile: one kernel on a fixed case, for profilers (profile_case)
    ap.add_argument("--kernel", default="spmv", choices=["spmv", "cg", "pcg", "bicgstab", "multi"])
    ap.add_argument("--prec", default=None, choices=["fp64", "mixed", "fp32", "fp16", "fp8"])
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--iters", type=int, default=50)
    ap.add_argument("--slab-bytes", type=int, default=0)
    ap.add_argument("--rb-per-slab", type=int, default=0)
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    ap.add_argument("--time", action="store_true")
    ap.add_argument("--trace", type=int, default=0)
    ap.add_argument("--prefetch", action="store_true")
    ap.add_argument("--no-tmem", action="store_true")
    ap.add_argument("--no-each", action="store_true", help="batch: skip the one-launch-per-system comparison")
    ap.add_argument("--batch-group", type=int, default=0, help="batch: CTAs per system group (0 = default)")
    args = ap.parse_args()
    if args.workload == "profile":
        profile_case(args)
        return
    world, rank, local, dist = _dist_setup(args)
    if args.impl == "reference":
        out = cpu_reference_arm(args, rank, world)
        if out is not None:
            print(json.dumps(out))
        return
    if args.workload in ("vs_cusparse", "multi16"):
        out = (cusparse_arm(args, rank, local) if args.workload == "vs_cusparse"
               else multi_rhs_arm(args, rank, local, fp64_panel=True))
        if out is not None:
            print(json.dumps(out))
        return
    if args.workload == "batch":
        out = batch_arm(args, world, rank, local, dist)
        if dist is not None:
            dist.barrier()
            dist.destroy_process_group()
        if out is not None:
            print(json.dumps(out))
        return
    out = gpu_arm(args, world, rank, local, dist)
    _extra_legs(args, world, rank, local, dist, out)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # one whole oracle solve (about 10 s of CPU work)
        a2 = argparse.Namespace(**vars(args))
        a2.steps, a2.warmup = 1, 0
        ref = cpu_reference_arm(a2, 0)
        out["cpu_baseline"] = ref["cpu_baseline"]
        sr = ref["cpu_baseline"].get("spmv_reference_1core", {})
        if "ms" in sr:
            out["spmv"]["fp64"]["speedup_vs_cpu_reference_1core"] = sr["ms"] / out["spmv"]["fp64"]["ms"]
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if out is not None:
        print(json.dumps(out))


if __name__ == "__main__":
    main()
