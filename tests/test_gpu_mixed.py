"""Mixed-precision layouts: per-tile precision from the magnitude rule,
bit-exact SpMV against the oracle's definition, and solves that reach the
FP64 true-residual tolerance."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_rule_layout_spmv_bitexact(mf, O):
    import torch

    for A in (mf.Matrix.varpoisson3d(24), mf.Matrix.poisson2d(96), mf.Matrix.spd_random(6000, 4)):
        n = A.n
        rp, ci, v = A.csr()
        t = mf.Tiles(A, mf.options(precision_mode=mf.MODE_MIXED_RULE))
        p, _ = t.precisions()
        assert p.max() > 0  # some tiles below FP64
        o = O.OracleTiles(n, n, rp, ci, v)
        x = np.random.default_rng(5).standard_normal(n)
        xd = torch.tensor(x, device="cuda")
        yd = torch.zeros(n, dtype=torch.float64, device="cuda")
        t.spmv_level_dev(0, xd.data_ptr(), yd.data_ptr())
        assert np.array_equal(yd.cpu().numpy(), o.mixed_spmv(p, x))


def test_random_low_precisions_bitexact(mf, O):
    """Every tile at a random precision below FP64 (FP32 / FP16 / FP8 class
    groups in one row block) on matrices whose row blocks keep their tiles."""
    import torch

    for A in (mf.Matrix.poisson2d(80), mf.Matrix.varpoisson3d(20)):
        n = A.n
        rp, ci, v = A.csr()
        t = mf.Tiles(A)
        p = np.random.default_rng(3).integers(1, 4, t.info()["tilenum"]).astype(np.uint8)
        t.set_precisions(p)
        pe, _ = t.precisions()
        assert np.array_equal(pe, p)
        x = np.random.default_rng(4).standard_normal(n)
        xd = torch.tensor(x, device="cuda")
        yd = torch.zeros(n, dtype=torch.float64, device="cuda")
        t.spmv_level_dev(0, xd.data_ptr(), yd.data_ptr())
        assert np.array_equal(yd.cpu().numpy(), O.OracleTiles(n, n, rp, ci, v).mixed_spmv(p, x))


def test_random_per_tile_precisions_bitexact(mf, O):
    """Planes whose entries come from tiles of different precisions / scales
    are stored at a common width without changing any dequantized value.
    A row block whose class groups need more than 32 planes in all is
    computed in FP64 from the tile arrays (its tiles report FP64), so the
    oracle takes the precisions the layout reports."""
    import torch

    A = mf.Matrix.spd_random(8000, 6)
    n = A.n
    rp, ci, v = A.csr()
    t = mf.Tiles(A)
    tn = t.info()["tilenum"]
    p = np.random.default_rng(1).integers(0, 4, tn).astype(np.uint8)
    t.set_precisions(p)
    pe, _ = t.precisions()
    assert np.all((pe == p) | (pe == 0)) and np.mean(pe == p) > 0.5
    o = O.OracleTiles(n, n, rp, ci, v)
    x = np.random.default_rng(2).standard_normal(n)
    xd = torch.tensor(x, device="cuda")
    yd = torch.zeros(n, dtype=torch.float64, device="cuda")
    t.spmv_level_dev(0, xd.data_ptr(), yd.data_ptr())
    y, yo = yd.cpu().numpy(), o.mixed_spmv(pe, x)
    bad = np.flatnonzero(y != yo)
    assert bad.size == 0, (bad[:8], y[bad[:4]], yo[bad[:4]])


@pytest.mark.parametrize("N", [24, 48])
def test_mixed_cg_reaches_fp64_tolerance(mf, N):
    A = mf.Matrix.varpoisson3d(N)
    b = A.b()
    t = mf.Tiles(A, mf.options(precision_mode=mf.MODE_MIXED_RULE))
    x64, r64 = t.solve_cg(b, tol=1e-10, maxiter=40000, opts=mf.options())
    xm, rm = t.solve_cg(b, tol=1e-10, maxiter=40000)
    assert r64["status"] == 0 and rm["status"] == 0, (r64, rm)
    assert rm["rel_residual_true"] <= 1e-10, rm
    assert rm["iterations"] <= 1.15 * r64["iterations"], (rm["iterations"], r64["iterations"])
    assert np.linalg.norm(xm - x64) / np.linalg.norm(x64) < 1e-6
    assert rm["replacements"] >= rm["iterations"] // 50


def test_mixed_cg_full_size_varpoisson_128(mf):
    A = mf.Matrix.varpoisson3d(128)
    b = A.b()
    t = mf.Tiles(A, mf.options(precision_mode=mf.MODE_MIXED_RULE))
    xm, rm = t.solve_cg(b, tol=1e-10, maxiter=40000)
    assert rm["status"] == 0 and rm["rel_residual_true"] <= 1e-10, rm
    xs = A.xstar()
    assert np.linalg.norm(xm - xs) / np.linalg.norm(xs) < 1e-4


@pytest.mark.parametrize("maker,growth", [("convdiff3d_24", 1.3), ("varpoisson3d_24", 1.7)])
def test_mixed_bicgstab_reaches_fp64_tolerance(mf, maker, growth):
    """BiCGSTAB on the low-precision layouts (FP64 vectors, dots and periodic
    true-residual replacement) reaches the FP64 true residual. On the
    contrast-1e6 Poisson (scaled condition ~1e8 at 24^3) the FP32 operator
    costs BiCGSTAB about 1.6x the FP64 iterations, CG only a few percent.
    BiCGSTAB runs FP32 tiles where the CG levels hold FP16 ones."""
    kind, size = maker.rsplit("_", 1)
    A = mf.Matrix.convdiff3d(int(size)) if kind == "convdiff3d" else mf.Matrix.varpoisson3d(int(size))
    b = A.b()
    t = mf.Tiles(A, mf.options(precision_mode=mf.MODE_MIXED_RULE))
    x64, r64 = t.solve_bicgstab(b, tol=1e-10, maxiter=20000, opts=mf.options())
    xm, rm = t.solve_bicgstab(b, tol=1e-10, maxiter=20000)
    assert r64["status"] == 0 and rm["status"] == 0, (r64, rm)
    assert rm["rel_residual_true"] <= 1e-10, rm
    assert sum(rm["iters_level"]) > 0  # iterations ran on a low-precision layout
    assert rm["iterations"] <= growth * r64["iterations"] + 5, (rm["iterations"], r64["iterations"])
    # both meet the 1e-10 residual; their difference is bounded by the
    # condition number times that, not by the rounding of either
    assert np.linalg.norm(xm - x64) / np.linalg.norm(x64) < 1e-5


def test_c3_mixed_layout_is_fp16_and_keeps_fp64_iterations(mf):
    """The headline matrix (diagonally dominant Z-matrix) is stored with
    row-sum-preserving FP16 tiles (diagonal entries FP32): the CG keeps the
    FP64 iteration count within a few percent and the FP64 true residual."""
    A = mf.Matrix.varpoisson3d(128)
    t = mf.Tiles(A, mf.options(precision_mode=mf.MODE_MIXED_RULE))
    x64, r64 = t.solve_cg(A.b(), tol=1e-10, maxiter=40000, opts=mf.options())
    xm, rm = t.solve_cg(A.b(), tol=1e-10, maxiter=40000)
    assert rm["status"] == 0 and rm["rel_residual_true"] <= 1e-10, rm
    assert rm["tile_frac"][2] > 0.99, rm["tile_frac"]
    assert rm["iterations"] <= 1.05 * r64["iterations"], (rm["iterations"], r64["iterations"])
    assert np.linalg.norm(xm - x64) / np.linalg.norm(x64) < 1e-6
    # the layout moves fewer bytes than an all-FP32 one would (FP16 values)
    assert rm["spmv_bytes_level"][0] < 0.8 * 113.5e6


def test_negative_row_sums_do_not_take_compensated_fp16(mf):
    """Row-sum compensation bounds the FP16 perturbation relative to the
    matrix only where the row sums are non-negative. A Z-matrix with negative
    row sums (the 2D Laplacian shifted by -0.5 lambda_min, still SPD) keeps
    the magnitude rule: no FP16 tiles. The unshifted Laplacian takes them."""
    N = 64
    A0 = mf.Matrix.poisson2d(N)
    rp, ci, v = A0.csr()
    rp, ci, v = np.asarray(rp), np.asarray(ci), np.asarray(v, dtype=np.float64).copy()
    lam_min = 4.0 - 4.0 * np.cos(np.pi / (N + 1))  # smallest eigenvalue of the 5-point Laplacian
    rows = np.repeat(np.arange(A0.n), np.diff(rp))
    v[ci == rows] -= 0.5 * lam_min
    A = mf.Matrix.from_csr(A0.n, A0.n, rp, ci, v)
    for M, want16 in ((A0, True), (A, False)):
        t = mf.Tiles(M, mf.options(precision_mode=mf.MODE_MIXED_RULE))
        _, r = t.solve_cg(np.ones(M.n), tol=1e-10, maxiter=20000)
        assert r["status"] == 0 and r["rel_residual_true"] <= 1e-10, r
        assert (r["tile_frac"][2] > 0.5) == want16, (want16, r["tile_frac"])


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["spd_random", "scattered"])
@pytest.mark.parametrize("tmem", [True, False])
def test_mixed_cg_fast_converging_systems(mf, case, tmem):
    """Diagonally dominant Z-matrices that CG solves in ~50-80 iterations
    (the batch workload's random SPD systems; a matrix of scattered columns,
    at most 4 entries a row) get compensated FP16 tiles. With so few
    iterations, the recursive residual reaches 1e-10 while the true residual
    still carries the FP16 operator's offset: the solve must restart its
    directions from the true residual at such a replacement instead of
    stagnating or diverging, and reach the FP64 true residual."""
    import sys
    import os

    sys.path.insert(0, os.path.dirname(__file__))
    from test_gpu_multi import _matching_spd

    if case == "spd_random":
        A = mf.Matrix.spd_random(30000, 5)
    else:
        M = _matching_spd(40000, 3, 9)
        A = mf.Matrix.from_csr(M.shape[0], M.shape[0], M.indptr, M.indices, M.data)
    b = np.random.default_rng(11).uniform(-1, 1, A.n)
    x64, r64 = mf.Tiles(A).solve_cg(b, tol=1e-10, maxiter=5000)
    t = mf.Tiles(A, mf.options(precision_mode=mf.MODE_MIXED_RULE))
    o = mf.options(precision_mode=mf.MODE_MIXED_RULE)
    if not tmem:
        o.reserved[5] = 1  # vectors in global memory (k_cgcg)
    x, r = t.solve_cg(b, tol=1e-10, maxiter=5000, opts=o)
    assert r["status"] == 0 and r["rel_residual_true"] <= 1e-10, r
    assert r["iterations"] <= 3 * r64["iterations"], (r["iterations"], r64["iterations"])
    assert np.linalg.norm(x - x64) / np.linalg.norm(x64) < 1e-7


@pytest.mark.gpu
@pytest.mark.parametrize("n", [5, 17, 33, 2047])
def test_mixed_solvers_on_tiny_systems(mf, n):
    """Mixed CG and BiCGSTAB on systems of fewer row blocks than CTAs (most
    CTAs own no rows) and ragged tails: the FP64 true residual at 1e-10 and
    the FP64 solver's solution."""
    import scipy.sparse as sp

    b = np.random.default_rng(n).uniform(-1, 1, n)
    for lo, hi in ((-1.0, -1.0), (-1.3, -0.7)):  # SPD for CG, nonsymmetric for BiCGSTAB
        rp, ci, v = [0], [], []
        for i in range(n):
            for j, a in ((i - 1, lo), (i, 2.5), (i + 1, hi)):
                if 0 <= j < n:
                    ci.append(j)
                    v.append(a)
            rp.append(len(ci))
        rp, ci, v = np.array(rp, np.int32), np.array(ci, np.int32), np.array(v)
        A = mf.Matrix.from_csr(n, n, rp, ci, v)
        M = sp.csr_matrix((v, ci, rp), shape=(n, n))
        t = mf.Tiles(A, mf.options(precision_mode=mf.MODE_MIXED_RULE))
        solve = t.solve_cg if lo == hi else t.solve_bicgstab
        x64, r64 = solve(b, tol=1e-10, maxiter=2000, opts=mf.options())
        xm, rm = solve(b, tol=1e-10, maxiter=2000)
        assert r64["status"] == 0 and rm["status"] == 0, (n, r64, rm)
        assert np.linalg.norm(b - M @ xm) / np.linalg.norm(b) <= 1.01e-10, (n, rm)
        assert np.linalg.norm(xm - x64) / np.linalg.norm(x64) < 1e-8, n
