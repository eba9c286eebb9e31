"""GPU encoder and tiled SpMV parity against the oracle and the golden
fixtures made from the reference's own code. Integer/byte arrays and the
FP64 SpMV must be bit-exact."""
import numpy as np
import pytest

from _oracle import ARRAY_SPECS

pytestmark = pytest.mark.gpu

DERIVED = ("nonzero_row_new", "tile_rowidx", "block_signal", "blockrowid_new", "blockcsr_ptr_new")


def _random(n, per_row, seed, unsorted=True, dense_rows=()):
    rng = np.random.default_rng(seed)
    rp, ci, va = [0], [], []
    for r in range(n):
        cols = set(rng.integers(0, n, size=int(rng.integers(0, per_row + 1))).tolist())
        cols.add(r)
        if r in dense_rows:
            cols |= set(range(n))
        cols = sorted(cols)
        if unsorted:
            rng.shuffle(cols)
        ci += cols
        va += rng.standard_normal(len(cols)).tolist()
        rp.append(len(ci))
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(va)


def _with_empty_rows(n, seed):
    rp, ci, va = _random(n, 5, seed)
    keep = np.ones(n, bool)
    keep[::7] = False  # empty rows
    rows = np.repeat(np.arange(n), np.diff(rp))
    m = keep[rows]
    counts = np.bincount(rows[m], minlength=n)
    return np.concatenate([[0], np.cumsum(counts)]).astype(np.int32), ci[m], va[m]


def _cases(mf):
    A = mf.Matrix.poisson2d(256)
    B = mf.Matrix.convdiff3d(64)
    C = mf.Matrix.varpoisson3d(32)
    D = mf.Matrix.spd_random(20000, 5)
    out = {"poisson2d_256": (A.n, *A.csr()), "convdiff3d_64": (B.n, *B.csr()),
           "varpoisson3d_32": (C.n, *C.csr()), "spd_random_20000": (D.n, *D.csr())}
    out["random_5000_unsorted"] = (5000, *_random(5000, 20, 1))
    out["dense_rows_4000"] = (4000, *_random(4000, 3, 2, dense_rows=(5, 6, 7, 3000)))  # >2048 per row block
    out["empty_rows_1001"] = (1001, *_with_empty_rows(1001, 3))
    return out


@pytest.fixture(scope="module")
def cases(mf):
    return _cases(mf)


def test_encoder_matches_golden(mf, golden):
    for case, g in golden.items():
        rowA, n = map(int, g["rowA"])
        rp = g["row_ptr"][: rowA + 1]
        nnz = int(rp[rowA])
        t = mf.Tiles(csr=(rowA, n, rp, g["col_idx"][:nnz], g["val"][:nnz]))
        ex = t.export()
        for name in ARRAY_SPECS:
            assert np.array_equal(ex[name], g[name]), (case, name)
        assert np.array_equal(ex["ptroffset1"], g["ptroffset1"]) and np.array_equal(ex["ptroffset2"], g["ptroffset2"])
        if rowA == n:
            y = t.spmv(g["x"])
            if rowA % 16 == 1:
                # Tile_create copies no values for a 1-row tail block
                # (csr2block.h:237-251), so the reference returns 0 there;
                # the device tiles keep the row and return the true product.
                assert np.array_equal(y[:-1], g["y"][:-1]) and g["y"][-1] == 0.0, case
                rp_, ci_, v_ = g["row_ptr"], g["col_idx"], g["val"]
                last = sum(v_[k] * g["x"][ci_[k]] for k in range(rp_[rowA - 1], rp_[rowA]))
                assert np.isclose(y[-1], last, rtol=1e-13, atol=1e-13), case
            else:
                assert np.array_equal(y, g["y"]), case


def test_encoder_matches_oracle(mf, O, cases):
    for name, (n, rp, ci, v) in cases.items():
        t = mf.Tiles(csr=(n, n, rp, ci, v))
        o = O.OracleTiles(n, n, rp, ci, v)
        ex = t.export()
        for k in ARRAY_SPECS:
            assert np.array_equal(ex[k], o.array(k)), (name, k)
        rc = o.row_compress()
        for k in DERIVED:
            assert np.array_equal(ex[k], rc[k]), (name, k)
        p1, p2, _ = o.offsets()
        assert np.array_equal(ex["ptroffset1"], p1) and np.array_equal(ex["ptroffset2"], p2), name


def test_spmv_bitexact_vs_oracle(mf, O, cases):
    rng = np.random.default_rng(0)
    for name, (n, rp, ci, v) in cases.items():
        t = mf.Tiles(csr=(n, n, rp, ci, v))
        o = O.OracleTiles(n, n, rp, ci, v)
        for _ in range(2):
            x = rng.standard_normal(n) * 10.0 ** rng.uniform(-3, 3, n)
            y = t.spmv(x)
            assert np.array_equal(y, o.spmv(x)), name


@pytest.mark.parametrize("slab_bytes,rb_per_slab", [(2048, 1), (4096, 3), (16384, 8), (0, 0)])
def test_spmv_small_slabs_and_fallback_modes(mf, O, cases, slab_bytes, rb_per_slab):
    """Tiny stages force many slabs per CTA, the gather mode and the
    oversize (global-memory) path; results stay bit-exact."""
    rng = np.random.default_rng(1)
    for name in ("poisson2d_256", "spd_random_20000", "dense_rows_4000", "empty_rows_1001"):
        n, rp, ci, v = cases[name]
        opts = mf.options(slab_bytes=slab_bytes, rb_per_slab=rb_per_slab)
        t = mf.Tiles(csr=(n, n, rp, ci, v), opts=opts)
        o = O.OracleTiles(n, n, rp, ci, v)
        x = rng.standard_normal(n)
        assert np.array_equal(t.spmv(x), o.spmv(x)), (name, slab_bytes)


@pytest.mark.parametrize("prec", [1, 2, 3])
def test_low_precision_spmv_bitexact_vs_oracle(mf, O, cases, prec):
    rng = np.random.default_rng(2)
    for name in ("poisson2d_256", "varpoisson3d_32", "spd_random_20000", "dense_rows_4000"):
        n, rp, ci, v = cases[name]
        t = mf.Tiles(csr=(n, n, rp, ci, v), opts=mf.options(precision_mode=mf.MODE_FIXED, fixed_precision=prec))
        o = O.OracleTiles(n, n, rp, ci, v)
        x = rng.standard_normal(n)
        import torch

        xd = torch.tensor(x, device="cuda")
        yd = torch.zeros(n, dtype=torch.float64, device="cuda")
        t.spmv_level_dev(0, xd.data_ptr(), yd.data_ptr())
        y = yd.cpu().numpy()
        p, _ = t.precisions()
        yo = o.mixed_spmv(p, x)
        assert np.array_equal(y, yo), (name, prec, np.max(np.abs(y - yo)))


def test_spmv_full_size_varpoisson_128(mf, O):
    A = mf.Matrix.varpoisson3d(128)
    n = A.n
    rp, ci, v = A.csr()
    t = mf.Tiles(A)
    inf = t.info()
    assert (inf["tilem"], inf["tilenum"]) == (131072, 880640)
    x = A.xstar()
    y = t.spmv(x)
    # b = A x* in CSR order differs from the tiled order only by rounding
    assert np.allclose(y, A.b(), rtol=1e-12, atol=1e-9)
    o = O.OracleTiles(n, n, rp, ci, v)
    assert np.array_equal(y, o.spmv(x))


def test_memory_report_tallies(mf):
    """The reference's memory-cost tallies for an FP64 and a mixed encoding,
    and the device bytes held by the handle."""
    A = mf.Matrix.varpoisson3d(20)
    n, nnz = A.n, A.nnz
    t64 = mf.Tiles(A)
    r = t64.memory_report()
    inf = t64.info()
    assert r["csr_bytes"] == (n + 1) * 4 + nnz * 12
    assert r["tile_value_bytes"] == [8.0 * nnz, 0.0, 0.0, 0.0]
    tn, tm = inf["tilenum"], inf["tilem"]
    idx = ((tm + 1) * 4 + tn * 4 + (tn + 1) + 2 * (tn + 1) * 4 + (tn + 3) * 4 + 2 * (inf["cnt_non_new"] + 1) + tn
           + nnz + tn * 4)
    assert r["tile_index_bytes"] == idx
    assert r["tile_total_bytes"] == idx + 8.0 * nnz
    assert r["slab_bytes_fp64"] == inf["layout_bytes"] and r["slab_bytes_mixed"] == 0
    assert r["device_bytes"] > r["slab_bytes_fp64"] + 8 * nnz
    tm_ = mf.Tiles(A, mf.options(precision_mode=mf.MODE_FIXED, fixed_precision=mf.PREC_FP16))
    rm = tm_.memory_report()
    assert rm["tile_value_bytes"] == [0.0, 0.0, 2.0 * nnz, 0.0]
    assert rm["slab_bytes_mixed"] > 0


@pytest.mark.parametrize("mode", ["fp64", "mixed"])
def test_autotune_keeps_results_and_picks_the_fastest(mf, mode):
    """The tuner times every slab geometry, leaves the handle on the fastest,
    and the SpMV and the solve give the same results afterwards."""
    import torch

    A = mf.Matrix.varpoisson3d(40)
    o = mf.options() if mode == "fp64" else mf.options(precision_mode=mf.MODE_MIXED_RULE)
    t = mf.Tiles(A, o)
    x = np.random.default_rng(8).standard_normal(A.n)
    xd = torch.tensor(x, device="cuda")
    y0 = torch.zeros_like(xd)
    y1 = torch.zeros_like(xd)
    level = -1 if mode == "fp64" else 0
    if level < 0:
        t.spmv_dev(xd.data_ptr(), y0.data_ptr())
    else:
        t.spmv_level_dev(0, xd.data_ptr(), y0.data_ptr())
    _, r0 = t.solve_cg(A.b(), tol=1e-10, maxiter=20000)
    tr = t.autotune(reps=10)
    assert len(tr["candidates"]) == 12
    assert tr["ms_best"] == min(c[2] for c in tr["candidates"]) and tr["ms_default"] > 0
    assert (tr["slab_bytes"], tr["rb_per_slab"]) in [(c[0], c[1]) for c in tr["candidates"]]
    if level < 0:
        t.spmv_dev(xd.data_ptr(), y1.data_ptr())
    else:
        t.spmv_level_dev(0, xd.data_ptr(), y1.data_ptr())
    assert torch.equal(y0, y1)  # bit-exact for every geometry
    _, r1 = t.solve_cg(A.b(), tol=1e-10, maxiter=20000)
    assert r1["status"] == 0 and r1["rel_residual_true"] <= 1e-10
    # the dot products' rounding follows the row-to-thread mapping, which the
    # slab grouping changes: iteration counts may move by a little
    assert abs(r1["iterations"] - r0["iterations"]) <= max(2, 0.02 * r0["iterations"])


@pytest.mark.parametrize("defect", ["col_high", "col_negative", "row_ptr_decreasing"])
def test_encode_rejects_invalid_csr(mf, defect):
    """The encoder checks the CSR on the GPU before any kernel indexes by it,
    for host (mf_encode) and device (mf_encode_dev) input alike."""
    import ctypes as C

    import torch

    A = mf.Matrix.poisson2d(16)
    rp, ci, v = A.csr()
    rp, ci, v = rp.astype(np.int32).copy(), ci.astype(np.int32).copy(), v.copy()
    if defect == "col_high":
        ci[len(ci) // 2] = A.n
    elif defect == "col_negative":
        ci[3] = -1
    else:
        rp[10], rp[11] = rp[11], rp[10]
    L = mf.lib()
    opts = mf.options()
    h = mf._p()
    csr = mf.MfCsr(A.n, A.n, len(v), rp.ctypes.data, ci.ctypes.data, v.ctypes.data)
    assert L.mf_encode(C.byref(csr), C.byref(opts), C.byref(h)) == mf.MF_ERR_ARG
    assert b"invalid CSR" in L.mf_last_error()
    drp, dci, dv = (torch.tensor(a, device="cuda") for a in (rp, ci, v))
    h2 = mf._p()
    rc = L.mf_encode_dev(A.n, A.n, len(v), C.c_void_p(drp.data_ptr()), C.c_void_p(dci.data_ptr()),
                         C.c_void_p(dv.data_ptr()), C.byref(opts), C.byref(h2))
    assert rc == mf.MF_ERR_ARG


@pytest.mark.parametrize("block_nnz", [64, 256, 2048])
def test_two_pointer_export_matches_oracle(mf, O, cases, block_nnz):
    """mf_balance_twopointer (the reference driver's warp work split, a
    compatibility export computed on the host from the handle's tile arrays)
    equals the oracle's restatement, unit for unit."""
    for name in ("poisson2d_256", "spd_random_20000", "dense_rows_4000"):
        n, rp, ci, v = cases[name]
        t = mf.Tiles(csr=(n, n, rp, ci, v))
        got = t.balance_twopointer(block_nnz, 180)
        want = O.OracleTiles(n, n, rp, ci, v).balance(block_nnz, 180)
        assert got[0] == want[0], (name, got[0], want[0])
        for g, w in zip(got[1:], want[1:]):
            assert np.array_equal(g, w), name
