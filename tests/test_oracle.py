"""The CPU oracle is pinned against the reference's own code: the golden
fixtures (made by tests/golden/make_golden.py from Tile_create and
blockspmv_cpu compiled unmodified) and, where the reference tree exists,
a live run of that code."""
import numpy as np
import pytest

from _oracle import ARRAY_SPECS


def test_oracle_matches_golden_tile_arrays(O, golden):
    for case, g in golden.items():
        rowA, n = map(int, g["rowA"])
        o = O.OracleTiles(rowA, n, g["row_ptr"], g["col_idx"], g["val"])
        for name in ARRAY_SPECS:
            assert np.array_equal(o.array(name), g[name]), (case, name)
        y = o.spmv(g["x"])
        assert np.array_equal(y, g["y"]), case  # bit-exact summation order
        p1, p2, rbb = o.offsets()
        assert np.array_equal(p1, g["ptroffset1"]) and np.array_equal(p2, g["ptroffset2"]), case
        assert rbb == int(g["rowblkblock"][0]), case


def _sym_random(n, seed):
    rng = np.random.default_rng(seed)
    import scipy.sparse as sp

    A = sp.random(n, n, density=min(1.0, 8.0 / n), random_state=seed, format="csr")
    A = (A + A.T + sp.identity(n) * 20).tocsr()
    A.sort_indices()
    return A


@pytest.mark.parametrize("n,seed", [(512, 0), (1000, 1), (4096, 2)])
def test_oracle_matches_reference_live(O, n, seed):
    if not O.ref_available():
        pytest.skip("reference harness not built (reference tree absent)")
    A = _sym_random(n, seed)
    o = O.OracleTiles(n, n, A.indptr, A.indices, A.data)
    r = O.RefTiles(n, n, A.indptr, A.indices, A.data)
    for name in ARRAY_SPECS:
        assert np.array_equal(o.array(name), r.array(name)), name
    x = np.random.default_rng(seed).standard_normal(n)
    assert np.array_equal(o.spmv(x), r.spmv(x)[0])


def test_reference_blockspmv_needs_nibble_columns(O, golden):
    """As shipped, blockspmv_cpu reads csr_compressedIdx, which Tile_create
    never fills; it is then exact only for x constant on each 16-segment.
    The oracle uses Tile_csr_Col (what the reference GPU kernels read)."""
    if not O.ref_available():
        pytest.skip("reference harness not built")
    g = golden["poisson2d_32"]
    rowA, n = map(int, g["rowA"])
    r = O.RefTiles(rowA, n, g["row_ptr"], g["col_idx"], g["val"])
    ones = np.ones(n)
    y0, *_ = r.spmv(ones, fill_compressed=False)
    o = O.OracleTiles(rowA, n, g["row_ptr"], g["col_idx"], g["val"])
    assert np.array_equal(y0, o.spmv(ones))


def test_oracle_cg_converges_and_matches_scipy(O):
    import scipy.sparse as sp

    A = _sym_random(2000, 3)
    b = np.random.default_rng(3).standard_normal(2000)
    o = O.OracleTiles(2000, 2000, A.indptr, A.indices, A.data)
    it, x, rel = O.OracleTiles.cg(o, b, 1e-10, 5000)
    assert rel <= 1e-10
    assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-9
    assert it > 5


def test_oracle_bicgstab_nonsymmetric(O):
    import scipy.sparse as sp

    rng = np.random.default_rng(4)
    A = sp.random(1500, 1500, density=0.004, random_state=4, format="csr") + sp.identity(1500) * 4
    A = A.tocsr()
    A.sort_indices()
    b = rng.uniform(-1, 1, 1500)
    o = O.OracleTiles(1500, 1500, A.indptr, A.indices, A.data)
    it, x, rel = o.bicgstab(b, 1e-10, 5000)
    assert rel <= 1e-10
    assert np.linalg.norm(b - A @ x) / np.linalg.norm(b) < 1e-9


def test_fp8_e4m3_encoding_spec(O):
    L = O.lib()
    # every code decodes and re-encodes to itself (except NaN)
    for code in range(256):
        v = L.mfo_fp8_e4m3_decode(code)
        if np.isnan(v):
            assert (code & 0x7F) == 0x7F
            continue
        enc = L.mfo_fp8_e4m3_encode(v)
        if v == 0.0:
            assert enc in (0x00, 0x80)
        else:
            assert enc == code, (code, v, enc)
    assert L.mfo_fp8_e4m3_decode(0x7E) == 448.0
    assert L.mfo_fp8_e4m3_encode(1e9) == 0x7E  # saturating
    assert L.mfo_fp8_e4m3_decode(0x01) == 2.0 ** -9
    # ties to even: 1 + 1/16 lies halfway between 1 and 1.125
    assert L.mfo_fp8_e4m3_decode(L.mfo_fp8_e4m3_encode(1.0625)) == 1.0
    assert L.mfo_fp8_e4m3_decode(L.mfo_fp8_e4m3_encode(1.1875)) == 1.25


def test_fp16_encoding_matches_numpy(O):
    L = O.lib()
    rng = np.random.default_rng(0)
    vals = np.concatenate([rng.standard_normal(2000) * 10.0 ** rng.integers(-8, 5, 2000), [65504.0, 6e-8, 1e-9]])
    for v in vals:
        h = L.mfo_fp16_encode(float(v))
        assert h == int(np.float16(v).view(np.uint16)), v


def test_two_pointer_balance_small_case(O):
    # 6 tiles with nnz [4, 1, 1, 1, 1, 4]: block_nnz 6, block_per_warp 180.
    # i=0 (4) joins; j=5: 4+4>=6 closes unit 1 with tiles {0,5};
    # i=1 (1) joins; j=4 (1) joins; i=2, j=3 (1,1) join -> last unit {1,4,2,3}.
    n = 96
    rp = [0]
    ci, va = [], []
    pattern = {0: [0, 1, 2, 3], 1: [4], 2: [5], 3: [5], 4: [5], 5: [5]}
    # one row block; tile k has the listed nnz in distinct column blocks
    entries = [(0, 0), (1, 0), (2, 0), (3, 0), (0, 16), (0, 32), (0, 48), (0, 64), (0, 80), (1, 80), (2, 80), (3, 80)]
    rows = {}
    for r, c in entries:
        rows.setdefault(r, []).append(c)
    for r in range(n):
        for c in sorted(rows.get(r, [])):
            ci.append(c)
            va.append(1.0)
        rp.append(len(ci))
    o = O.OracleTiles(16, n, np.array(rp[:17]), np.array(ci), np.array(va))
    idx, bp, a, b, c = o.balance(6, 180)
    assert list(o.array("blknnz")) == [0, 4, 5, 6, 7, 8, 12]
    assert idx == 2
    assert list(bp) == [0, 2, 6]
    assert list(a[:6]) == [0, 5, 1, 4, 2, 3]


def _np_mlp_grad(w, x, y):
    """FP64 numpy forward/backward of the 6-64-64-4 ReLU MLP (softmax
    cross-entropy, mean over the batch): an independent check of the oracle."""
    w = w.astype(np.float64)
    W1, b1 = w[0:384].reshape(64, 6), w[384:448]
    W2, b2 = w[448:4544].reshape(64, 64), w[4544:4608]
    W3, b3 = w[4608:4864].reshape(4, 64), w[4864:4868]
    x = x.astype(np.float64)
    z1 = x @ W1.T + b1
    h1 = np.maximum(z1, 0)
    z2 = h1 @ W2.T + b2
    h2 = np.maximum(z2, 0)
    o = h2 @ W3.T + b3
    o -= o.max(1, keepdims=True)
    p = np.exp(o)
    p /= p.sum(1, keepdims=True)
    n = len(x)
    loss = -np.mean(np.log(p[np.arange(n), y]))
    d3 = p.copy()
    d3[np.arange(n), y] -= 1
    d3 /= n
    d2 = (d3 @ W3) * (z2 > 0)
    d1 = (d2 @ W2) * (z1 > 0)
    g = np.concatenate([(d1.T @ x).ravel(), d1.sum(0), (d2.T @ h1).ravel(), d2.sum(0), (d3.T @ h2).ravel(),
                        d3.sum(0)])
    return g, loss


def test_oracle_mlp_gradient_matches_numpy(O):
    rng = np.random.default_rng(12)
    w = (rng.standard_normal(4868) * 0.3).astype(np.float32)
    x = rng.standard_normal((300, 6)).astype(np.float32)
    y = rng.integers(0, 4, 300)
    g, loss = O.mlp_grad(w, x, y)
    g64, loss64 = _np_mlp_grad(w, x, y)
    assert abs(loss - loss64) <= 1e-5 * loss64
    assert np.linalg.norm(g - g64) <= 1e-4 * np.linalg.norm(g64)
    logits = O.mlp_forward(w, x)
    assert logits.shape == (300, 4)


def test_oracle_jacobi_pcg_solves_and_beats_cg_on_contrast(O):
    """The PCG restatement reaches the tolerance with the true residual, and on
    a high-contrast variable-coefficient Poisson needs far fewer iterations
    than CG (what Jacobi scaling is for)."""
    import importlib

    mf = importlib.import_module("mille-feillue_b200")
    A = mf.Matrix.varpoisson3d(12, 1e-3, 1e3, 4)
    n = A.n
    rp, ci, v = A.csr()
    diag = np.zeros(n)
    for i in range(n):
        cols = ci[rp[i]:rp[i + 1]]
        diag[i] = v[rp[i]:rp[i + 1]][cols == i].sum()
    o = O.OracleTiles(n, n, rp, ci, v)
    b = A.b()
    it_p, x_p, rel_p = o.pcg_jacobi(diag, b, 1e-10, 20000)
    it_c, _, _ = o.cg(b, 1e-10, 20000)
    import scipy.sparse as sp

    M = sp.csr_matrix((v, ci, rp), shape=(n, n))
    assert rel_p <= 1e-10
    assert np.linalg.norm(b - M @ x_p) / np.linalg.norm(b) <= 2e-10
    assert it_p < 0.5 * it_c, (it_p, it_c)


def test_mixed_operator_preserves_row_sums(O):
    """Row-sum-preserving compensation: with every tile in FP16 (diagonal
    entries promoted to FP32), A~ 1 equals A 1 up to the FP32 rounding of
    the diagonal and of the row's FP32 accumulation; without it the FP16
    rounding of the off-diagonals (relative 4.9e-4) would show."""
    S = O.gen_varpoisson3d(12)
    rp, ci, v = S.csr()
    o = O.OracleTiles(S.n, S.n, rp, ci, v)
    prec = np.full(o.sizes["tilenum"], 2, np.uint8)
    ones = np.ones(S.n)
    y = o.mixed_spmv(prec, ones)
    rows = np.repeat(np.arange(S.n), np.diff(rp))
    rowsum = np.bincount(rows, weights=v, minlength=S.n)
    absum = np.bincount(rows, weights=np.abs(v), minlength=S.n)
    err = np.abs(y - rowsum)
    assert np.all(err <= 16 * 2.0 ** -24 * absum), (err / absum).max()
    # the compensated diagonal is what carries it: the off-diagonal FP16
    # rounding alone is orders of magnitude larger than the error left
    off = ci != rows
    h = v[off].astype(np.float16).astype(np.float64)  # the tile scales are powers of two
    assert np.abs(h - v[off]).max() > 100 * err.max()


def test_mixed_operator_keeps_non_z_rows_uncompensated(O):
    """A row with a positive off-diagonal entry keeps its diagonal's plain
    class value: A~ 1 then differs from A 1 by the off-diagonals' rounding."""
    n = 64
    rp = np.arange(0, 3 * n + 1, 3, dtype=np.int32)[: n + 1]
    ci, v = [], []
    for i in range(n):
        cols = sorted({i, (i + 1) % n, (i + 7) % n})
        while len(cols) < 3:
            cols.append((cols[-1] + 1) % n)
        for c in cols:
            ci.append(c)
            v.append(10.0 if c == i else 0.1 + 0.001 * (i % 13))  # positive off-diagonals
    ci = np.array(ci, np.int32)
    v = np.array(v)
    o = O.OracleTiles(n, n, rp, ci, v)
    prec = np.full(o.sizes["tilenum"], 2, np.uint8)
    y = o.mixed_spmv(prec, np.ones(n))
    rows = np.repeat(np.arange(n), 3)
    # compensation would make y equal the FP64 row sums to FP32 accuracy;
    # rows that are not Z-rows keep the FP16 rounding of their off-diagonals
    rs = np.bincount(rows, weights=v, minlength=n)
    assert np.max(np.abs(y - rs)) > 4 * 2.0 ** -24 * np.max(np.abs(rs))
