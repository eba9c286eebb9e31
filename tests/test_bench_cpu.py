"""CPU legs of bench.py: the reference's own serial tiled SpMV timing
returns a well-formed record (and its product is the oracle's), the CPU
solves of the two smaller configurations reach the tolerance, and the
reference arm times whole oracle solves without loading the product
library."""
import json
import os
import subprocess
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_cpu_spmv_reference_record(mf, O):
    import bench

    A = mf.Matrix.varpoisson3d(16)
    rp, ci, v = A.csr()
    r = bench._cpu_spmv_reference(O, A.n, rp, ci, v, A.xstar())
    if "unavailable" in r:  # the reference sources were absent at build time
        return
    assert r["kind"] == "reference" and r["cores"] == 1 and r["ms"] > 0
    # FP64 values + 1-byte columns per entry, 8 B per tile, x read and y written
    tiles = O.RefTiles(A.n, A.n, rp, ci, v)
    assert r["alg_bytes"] == 9.0 * len(v) + 8.0 * tiles.sizes["tilenum"] + 16.0 * A.n
    y, _, _, _ = tiles.spmv(A.xstar())
    assert np.array_equal(y, O.OracleTiles(A.n, A.n, rp, ci, v).spmv(A.xstar()))


def test_cpu_small_configs(mf, O):
    import bench

    r = bench._cpu_small_configs(O)
    assert set(r) == {"C1_poisson2d_256_cg", "C2_convdiff3d_64_bicgstab"}
    for v in r.values():
        assert v["ms"] > 0 and v["iterations"] > 0 and v["rel_residual"] <= bench.TOL


_ARM = r"""
import argparse, json, sys
sys.path.insert(0, {root!r})
import bench
a = argparse.Namespace(gpus=1, steps=2, warmup=1, grid=16)
out = bench.cpu_reference_arm(a, 0, 1, small=False)
maps = open("/proc/self/maps").read()
out["_libmf_mapped"] = "libmf.so" in maps
out["_product_imported"] = "mille-feillue_b200" in sys.modules
print(json.dumps(out))
"""


def test_reference_arm_times_whole_solves_without_the_product():
    p = subprocess.run([sys.executable, "-c", _ARM.format(root=ROOT)], capture_output=True, text=True, timeout=300,
                       cwd=ROOT)
    assert p.returncode == 0, p.stderr[-2000:]
    r = json.loads(p.stdout.strip().splitlines()[-1])
    assert not r["_libmf_mapped"] and not r["_product_imported"]
    assert r["impl"] == "reference" and r["steps"] == 2 and r["warmup"] == 1
    cb = r["cpu_baseline"]
    assert cb["kind"] == "port" and cb["iterations"] > 0 and cb["rel_residual"] <= 1e-10
    assert cb["step_ms_min_max"][0] <= r["value"] <= cb["step_ms_min_max"][1]
    assert r["config"]["n"] == 16 ** 3 and r["config"]["nnz"] == 7 * 16 ** 3 - 6 * 16 ** 2


def test_both_arms_share_the_config():
    import bench

    c = bench._config(1, 128)
    assert c == bench._config(1, 128) and c["n"] == 2097152 and c["nnz"] == 14581760
    assert bench._config(2, 128)["parallelism"] == "replicas"
