"""CPU legs of bench.py: the reference's own serial tiled SpMV timing
returns a well-formed record (and its product is the oracle's), and the CPU
solves of the two smaller configurations reach the tolerance."""
import numpy as np


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

    r = bench._cpu_small_configs(O, mf)
    assert set(r) == {"C1_poisson2d_256_cg", "C2_convdiff3d_64_bicgstab"}
    for v in r.values():
        assert v["ms"] > 0 and v["iterations"] > 0 and v["rel_residual"] <= bench.TOL
