"""SuiteSparse sweep driver: the counterpart of Performance-Comparison/test.sh.

For every (name, nnz) row of a dataset CSV in the layout of the reference's
CG_dataset.csv / BiCGSTAB_dataset.csv, the sweep finds <name>.mtx under the
matrix root (recursively, as test.sh's `find` does) and runs the drop-in
drivers bin/Mille-feuille_CG_NVIDIA and bin/Mille-feuille_BiCGSTAB_NVIDIA on
it with the reference's argv (`matrix.mtx [block_nnz]`). Each driver prints
one result line (`iter=..,time_cg=.. ms,rel_residual=..,true_rel_residual=..`);
the sweep collects them, one CSV row per matrix and solver.

    python mille-feillue_b200/sweep.py CG_dataset.csv /home/dataset/MM --out sweep_cg.csv
    python mille-feillue_b200/sweep.py BiCGSTAB_dataset.csv /home/dataset/MM --solvers bicgstab

The SuiteSparse matrices themselves are not part of this repository; any
directory of Matrix Market files works. Matrices that are not found are
recorded with status "missing"; a driver that fails or runs past the
per-run timeout is recorded with its status.
"""
import argparse
import csv
import os
import re
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
DRIVERS = {"cg": os.path.join(HERE, "bin", "Mille-feuille_CG_NVIDIA"),
           "bicgstab": os.path.join(HERE, "bin", "Mille-feuille_BiCGSTAB_NVIDIA")}
RESULT = re.compile(r"iter=(?P<iter>-?\d+),time_(?:cg|bicg)=(?P<ms>[-+0-9.eE]+) ms,"
                    r"rel_residual=(?P<rel>[-+0-9.eEnaif]+),true_rel_residual=(?P<true>[-+0-9.eEnaif]+)")
FIELDS = ["name", "nnz_class", "solver", "status", "iterations", "time_ms", "rel_residual",
          "true_rel_residual", "path"]


def read_dataset(path):
    """(name, nnz) rows of a dataset CSV with a header line, as test.sh reads them."""
    rows = []
    with open(path, newline="") as f:
        r = csv.reader(f)
        next(r, None)  # header
        for rec in r:
            if rec and rec[0].strip():
                rows.append((rec[0].strip(), rec[1].strip() if len(rec) > 1 else ""))
    return rows


def find_matrices(root, name):
    hits = []
    for d, _, files in os.walk(root):
        if name + ".mtx" in files:
            hits.append(os.path.join(d, name + ".mtx"))
    return sorted(hits)


def parse_result(text):
    m = RESULT.search(text)
    if not m:
        return None
    return {"iterations": int(m["iter"]), "time_ms": float(m["ms"]), "rel_residual": float(m["rel"]),
            "true_rel_residual": float(m["true"])}


def run_one(solver, path, block_nnz, timeout):
    argv = [DRIVERS[solver], path] + ([str(block_nnz)] if block_nnz else [])
    try:
        p = subprocess.run(argv, capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return {"status": "timeout"}
    res = parse_result(p.stdout)
    if p.returncode != 0 or res is None:
        if "unequal" in p.stdout:
            return {"status": "not square"}
        return {"status": f"error rc={p.returncode}"}
    res["status"] = "ok"
    return res


def sweep(dataset, root, solvers, out, block_nnz=0, timeout=600):
    for s in solvers:
        if not os.path.exists(DRIVERS[s]):
            raise SystemExit(f"driver not built: {DRIVERS[s]} (run __graft_entry__.build())")
    rows = []
    with open(out, "w", newline="") as f:
        w = csv.DictWriter(f, fieldnames=FIELDS)
        w.writeheader()
        for name, nnz in read_dataset(dataset):
            paths = find_matrices(root, name) if os.path.isdir(root) else []
            if not paths:
                for s in solvers:
                    row = {"name": name, "nnz_class": nnz, "solver": s, "status": "missing", "path": ""}
                    w.writerow(row)
                    rows.append(row)
                continue
            for path in paths:
                for s in solvers:
                    row = {"name": name, "nnz_class": nnz, "solver": s, "path": path}
                    row.update(run_one(s, path, block_nnz, timeout))
                    w.writerow(row)
                    f.flush()
                    rows.append(row)
    return rows


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("dataset", help="CSV with a header and rows name,nnz (CG_dataset.csv layout)")
    ap.add_argument("root", help="directory searched recursively for <name>.mtx")
    ap.add_argument("--out", default="sweep.csv")
    ap.add_argument("--solvers", default="cg,bicgstab")
    ap.add_argument("--block-nnz", type=int, default=0, help="passed to the drivers as their second argument")
    ap.add_argument("--timeout", type=float, default=600.0, help="seconds per driver run")
    a = ap.parse_args(argv)
    solvers = [s for s in a.solvers.split(",") if s]
    for s in solvers:
        if s not in DRIVERS:
            raise SystemExit(f"unknown solver {s}")
    rows = sweep(a.dataset, a.root, solvers, a.out, a.block_nnz, a.timeout)
    ok = sum(r["status"] == "ok" for r in rows)
    print(f"{ok} of {len(rows)} runs ok -> {a.out}")
    return 0


if __name__ == "__main__":
    sys.exit(main())
