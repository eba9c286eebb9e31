"""Generates tests/golden/configs_oracle.json: full FP64 solves by the CPU
oracle (restatement of the reference recurrences, tiled SpMV in the
reference's order) of the measured configurations, on matrices built by
the oracle's own generators:

  C1  CG on the 2D 5-point Poisson 256^2 (b = A * ones)
  C2  BiCGSTAB on the 3D convection-diffusion 64^3 (b ~ U[-1, 1], seed 0)
  C3  CG and Jacobi-PCG on the 3D variable-coefficient Poisson 128^3
      (faces logU[1e-3, 1e3], seed 1; b = A x*)

all from x0 = 0 to a 1e-10 relative residual. For each: the iteration
count, the final residual, ||x - x*|| / ||x*|| where x* exists, and x at
1024 evenly spaced rows. The C3 solves take about 10-20 s each on a few
host cores, so the GPU tests read these numbers instead of re-running them.

Run from the repository root after `make -C oracle`:
    python tests/golden/make_configs.py
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import _oracle as O  # noqa: E402

TOL = 1e-10
SAMPLES = 1024


def _record(S, solver, extra=None):
    o = O.OracleTiles(S.n, S.n, *S.csr())
    t0 = time.perf_counter()
    if solver == "pcg_jacobi":
        it, x, rel = o.pcg_jacobi(extra, S.b, TOL, 40000)
    else:
        it, x, rel = getattr(o, solver)(S.b, TOL, 40000)
    dt = time.perf_counter() - t0
    idx = np.linspace(0, S.n - 1, SAMPLES).astype(np.int64)
    rec = {"n": S.n, "nnz": int(S.ci.size), "solver": solver, "iterations": int(it), "rel_residual": float(rel),
           "sample_rows": idx.tolist(), "x_sample": x[idx].tolist(), "oracle_seconds": dt}
    if S.xstar is not None:
        rec["x_err_vs_xstar"] = float(np.linalg.norm(x - S.xstar) / np.linalg.norm(S.xstar))
    return rec


def _diag(S):
    rows = np.repeat(np.arange(S.n), np.diff(S.rp))
    d = np.zeros(S.n)
    np.add.at(d, rows[S.ci == rows], S.v[S.ci == rows])
    return d


def main():
    O.set_threads(len(os.sched_getaffinity(0)))
    out = {"tol": TOL}
    out["C1_poisson2d_256_cg"] = _record(O.gen_poisson2d(256), "cg")
    out["C2_convdiff3d_64_bicgstab"] = _record(O.gen_convdiff3d(64), "bicgstab")
    S = O.gen_varpoisson3d(128)
    out["C3_varpoisson3d_128_cg"] = _record(S, "cg")
    out["C3_varpoisson3d_128_pcg_jacobi"] = _record(S, "pcg_jacobi", _diag(S))
    with open(os.path.join(HERE, "configs_oracle.json"), "w") as f:
        json.dump(out, f, indent=1)
    for k, v in out.items():
        if isinstance(v, dict):
            print(k, v["iterations"], v["rel_residual"], round(v["oracle_seconds"], 2))


if __name__ == "__main__":
    main()
