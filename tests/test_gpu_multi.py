"""CG on up to 16 right-hand sides at once: every column against the
single-right-hand-side solver and the CPU oracle's CG."""
import numpy as np
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("k", [16, 5])
def test_multi_rhs_fp64_panel_columns_match_single_solves(mf, O, k):
    """MF_PANEL_FP64: every column is the single-right-hand-side FP64 CG."""
    import scipy.sparse as sp

    A = mf.Matrix.varpoisson3d(16)
    n = A.n
    rp, ci, v = A.csr()
    rng = np.random.default_rng(20 + k)
    B = rng.uniform(-1, 1, (n, k))
    B[:, 0] = A.b()
    X, it, rel, ms = mf.solve_cg_multi(A, B, tol=1e-10, maxiter=20000, panel=mf.PANEL_FP64)
    assert ms > 0
    M = sp.csr_matrix((v, ci, rp), shape=(n, n))
    t = mf.Tiles(A)
    o = O.OracleTiles(n, n, rp, ci, v)
    for j in range(k):
        b = B[:, j]
        assert rel[j] <= 1e-10
        assert np.linalg.norm(b - M @ X[:, j]) / np.linalg.norm(b) <= 2e-10
        xs, rs = t.solve_cg(b, tol=1e-10, maxiter=20000)
        assert abs(int(it[j]) - rs["iterations"]) <= max(2, 0.02 * rs["iterations"]), (j, it[j], rs["iterations"])
        assert np.linalg.norm(X[:, j] - xs) / np.linalg.norm(xs) < 1e-8
        if j < 2:
            it_o, _, _ = o.cg(b, 1e-10, 20000)
            assert abs(int(it[j]) - it_o) <= max(2, 0.02 * it_o)


@pytest.mark.gpu
@pytest.mark.parametrize("k", [16, 3])
def test_multi_rhs_fp32_panel_columns_match_oracle(mf, O, k):
    """MF_PANEL_FP32 (the persistent kernel): each column against the
    oracle's FP32-direction CG (mfo_cg_dir32, the same recurrence summed in
    another order): iterations within 2 %, the FP64 true residual at tol,
    and x against the oracle's and the FP64 CG's solutions."""
    import scipy.sparse as sp

    A = mf.Matrix.varpoisson3d(16)
    n = A.n
    rp, ci, v = A.csr()
    rng = np.random.default_rng(40 + k)
    B = rng.uniform(-1, 1, (n, k))
    B[:, 0] = A.b()
    X0 = np.zeros((n, k))
    X0[:, -1] = rng.uniform(-1, 1, n)  # one column starts from a non-zero x0
    X, it, rel, ms = mf.solve_cg_multi(A, B, X0=X0, tol=1e-10, maxiter=20000)
    assert ms > 0
    M = sp.csr_matrix((v, ci, rp), shape=(n, n))
    o = O.OracleTiles(n, n, rp, ci, v)
    for j in range(k):
        b = B[:, j]
        true_rel = np.linalg.norm(b - M @ X[:, j]) / np.linalg.norm(b)
        assert rel[j] <= 1e-10 and true_rel <= 1.01e-10, (j, rel[j], true_rel)
        it_o, x_o, rel_o = o.cg_dir32(b, 1e-10, 20000, replace=50, x0=X0[:, j])
        assert rel_o <= 1e-10
        assert abs(int(it[j]) - it_o) <= max(2, 0.02 * it_o), (j, it[j], it_o)
        assert np.linalg.norm(X[:, j] - x_o) / np.linalg.norm(x_o) < 1e-7
        it64, x64, _ = o.cg(b, 1e-10, 20000, x0=X0[:, j])
        assert np.linalg.norm(X[:, j] - x64) / np.linalg.norm(x64) < 1e-7
        assert it[j] <= 1.06 * it64, (j, it[j], it64)


@pytest.mark.gpu
def test_multi_rhs_fp32_panel_at_64_cubed_keeps_fp64_iterations(mf):
    """k = 16 on the 64^3 variable-coefficient Poisson: the FP32 panels
    reach the 1e-10 true residual in every column within 3 % of the FP64
    panel's iterations (speed is measured by the benchmark at 128^3)."""
    import scipy.sparse as sp

    A = mf.Matrix.varpoisson3d(64)
    n = A.n
    rp, ci, v = A.csr()
    B = np.random.default_rng(3).uniform(-1, 1, (n, 16))
    X32, it32, rel32, ms32 = mf.solve_cg_multi(A, B, tol=1e-10, maxiter=40000)
    X64, it64, rel64, ms64 = mf.solve_cg_multi(A, B, tol=1e-10, maxiter=40000, panel=mf.PANEL_FP64)
    M = sp.csr_matrix((v, ci, rp), shape=(n, n))
    for j in range(16):
        assert rel32[j] <= 1e-10 and rel64[j] <= 1e-10
        assert np.linalg.norm(B[:, j] - M @ X32[:, j]) / np.linalg.norm(B[:, j]) <= 1.01e-10
        assert it32[j] <= 1.03 * it64[j], (j, it32[j], it64[j])
        assert np.linalg.norm(X32[:, j] - X64[:, j]) / np.linalg.norm(X64[:, j]) < 1e-6


def test_multi_rhs_argument_checks(mf):
    import ctypes as C

    A = mf.Matrix.poisson2d(8)
    n = A.n
    B = np.zeros((n, 17), order="F")
    X = np.zeros((n, 17), order="F")
    it = np.zeros(17, np.int32)
    rel = np.zeros(17)
    ms = C.c_double()
    rc = mf.lib().mf_solve_cg_multi(C.byref(A.csr_struct()), 17, mf._ptr(B), mf._ptr(X), 1e-10, 10, mf._ptr(it),
                                    mf._ptr(rel), C.byref(ms))
    assert rc == mf.MF_ERR_ARG
    rp, ci, v = A.csr()
    ci2 = ci.copy()
    ci2[rp[1]:rp[2]] = ci2[rp[1]:rp[2]][::-1]  # a row with descending columns
    U = mf.Matrix.from_csr(n, n, rp, ci2, v)
    rc = mf.lib().mf_solve_cg_multi(C.byref(U.csr_struct()), 2, mf._ptr(B), mf._ptr(X), 1e-10, 10, mf._ptr(it),
                                    mf._ptr(rel), C.byref(ms))
    assert rc == mf.MF_ERR_ARG
    assert b"ascend" in mf.lib().mf_last_error()


def _dev_multi(mf, n, rp, ci, v, B, tol=1e-10, maxiter=20000):
    import ctypes as C

    import torch

    k = B.shape[1]
    d = lambda a: torch.tensor(np.ascontiguousarray(a), device="cuda")
    rpd, cid, vd = d(np.asarray(rp, np.int32)), d(np.asarray(ci, np.int32)), d(np.asarray(v, np.float64))
    Bd = d(np.asfortranarray(B).T.reshape(-1))  # column-major n x k
    Xd = torch.zeros_like(Bd)
    it = np.zeros(k, np.int32)
    rel = np.zeros(k)
    ms = C.c_double()
    rc = mf.lib().mf_solve_cg_multi_dev(n, rpd.data_ptr(), cid.data_ptr(), vd.data_ptr(), k, Bd.data_ptr(),
                                        Xd.data_ptr(), tol, maxiter, mf._ptr(it), mf._ptr(rel), C.byref(ms))
    torch.cuda.synchronize()
    return rc, Xd.cpu().numpy().reshape(k, n).T, it, rel


@pytest.mark.gpu
def test_multi_rhs_long_rows_use_csr_loop(mf):
    """An arrow matrix (first row and column full, 300 entries) is longer
    than the padded copy takes: the CSR loop solves it."""
    import scipy.sparse as sp

    n = 300
    rng = np.random.default_rng(5)
    D = np.diag(np.full(n, 2.0 * n))
    D[0, 1:] = rng.uniform(-1, 0, n - 1)
    D[1:, 0] = D[0, 1:]
    A = sp.csr_matrix(D)
    A.sort_indices()
    B = rng.uniform(-1, 1, (n, 3))
    rc, X, it, rel = _dev_multi(mf, n, A.indptr, A.indices, A.data, B)
    assert rc == 0, mf.lib().mf_last_error()
    for j in range(3):
        assert np.linalg.norm(B[:, j] - A @ X[:, j]) / np.linalg.norm(B[:, j]) <= 2e-10


@pytest.mark.gpu
def test_multi_rhs_dev_rejects_invalid_csr(mf):
    A = mf.Matrix.poisson2d(8)
    n = A.n
    rp, ci, v = A.csr()
    B = np.ones((n, 2))
    bad_col = ci.copy()
    bad_col[5] = n
    rc, _, _, _ = _dev_multi(mf, n, rp, bad_col, v, B, maxiter=10)
    assert rc == mf.MF_ERR_ARG and b"outside" in mf.lib().mf_last_error()
    bad_rp = rp.copy()
    bad_rp[3] = bad_rp[4] + 1
    rc, _, _, _ = _dev_multi(mf, n, bad_rp, ci, v, B, maxiter=10)
    assert rc == mf.MF_ERR_ARG and b"row_ptr" in mf.lib().mf_last_error()
    desc = ci.copy()
    desc[rp[1]:rp[2]] = desc[rp[1]:rp[2]][::-1]
    rc, _, _, _ = _dev_multi(mf, n, rp, desc, v, B, maxiter=10)
    assert rc == mf.MF_ERR_ARG and b"ascend" in mf.lib().mf_last_error()
    # the valid matrix still solves through the same entry point
    rc, X, _, rel = _dev_multi(mf, n, rp, ci, v, B)
    assert rc == 0 and rel.max() <= 1e-10


def _matching_spd(n, k, seed):
    """Symmetric, strictly diagonally dominant matrix whose off-diagonal
    pattern is the union of k random perfect matchings: at most k + 1
    entries a row, columns scattered over the whole matrix."""
    import scipy.sparse as sp

    rng = np.random.default_rng(seed)
    rows, cols, vals = [], [], []
    for _ in range(k):
        perm = rng.permutation(n)
        a, b = perm[0::2], perm[1::2]
        w = -rng.uniform(0.1, 1.0, len(a))
        rows += [a, b]
        cols += [b, a]
        vals += [w, w]
    M = sp.csr_matrix((np.concatenate(vals), (np.concatenate(rows), np.concatenate(cols))), shape=(n, n))
    M = M + sp.diags(np.asarray(abs(M).sum(1)).ravel() + 0.05)
    M = sp.csr_matrix(M)
    M.sort_indices()
    return M


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["scattered_8", "random_spd_pad32"])
def test_multi_rhs_fp32_panel_other_product_modes(mf, O, case):
    """The persistent panel kernel's other product modes against the oracle:
    a matrix of at most 8 entries a row whose 128-row blocks reach too many
    panel segments to stage (window mode, unstaged blocks: panel rows loaded
    from global memory), and the random SPD systems of the batch workload
    (~17 entries a row, padded to 32: the padded-gather mode with per-thread
    asynchronous copies). Every column: iterations within 2 % (or 2) of the
    oracle's FP32-direction CG, the FP64 true residual at tol, x within 1e-7
    of the oracle's."""
    import scipy.sparse as sp

    if case == "scattered_8":
        M = _matching_spd(40000, 3, 9)
        assert np.diff(M.indptr).max() <= 8
        A = mf.Matrix.from_csr(M.shape[0], M.shape[0], M.indptr, M.indices, M.data)
    else:
        A = mf.Matrix.spd_random(30000, 5)
        rp, ci, v = A.csr()
        M = sp.csr_matrix((v, ci, rp), shape=(A.n, A.n))
        assert 8 < np.diff(rp).max() <= 64
    n = A.n
    rp, ci, v = A.csr()
    B = np.random.default_rng(11).uniform(-1, 1, (n, 16))
    X, it, rel, _ = mf.solve_cg_multi(A, B, tol=1e-10, maxiter=5000)
    o = O.OracleTiles(n, n, rp, ci, v)
    for j in range(16):
        b = B[:, j]
        assert rel[j] <= 1e-10
        assert np.linalg.norm(b - M @ X[:, j]) / np.linalg.norm(b) <= 1.01e-10
        if j % 5 == 0:
            it_o, x_o, rel_o = o.cg_dir32(b, 1e-10, 5000)
            assert rel_o <= 1e-10
            assert abs(int(it[j]) - it_o) <= max(2, 0.02 * it_o), (j, it[j], it_o)
            assert np.linalg.norm(X[:, j] - x_o) / np.linalg.norm(x_o) < 1e-7


def _band_spd(n, half):
    """SPD band matrix: -1 on the `half` diagonals each side, diagonal
    2 * half + 1 (strictly diagonally dominant)."""
    rp, ci, v = [0], [], []
    for i in range(n):
        for j in range(max(0, i - half), min(n, i + half + 1)):
            ci.append(j)
            v.append(2.0 * half + 1.0 if j == i else -1.0)
        rp.append(len(ci))
    return np.array(rp, np.int32), np.array(ci, np.int32), np.array(v)


@pytest.mark.gpu
@pytest.mark.parametrize("case", ["band_17_csr", "varpoisson3d_3_win", "poisson2d_10_win", "band_50_pad"])
@pytest.mark.parametrize("panel", ["fp32", "fp64"])
def test_multi_rhs_tiny_systems(mf, case, panel):
    """Systems smaller than one 128-row block (most CTAs own no rows; the
    panels are padded to a whole block) in each product mode: CSR rows
    (W = 3), 128-row windows (W = 8), padded rows (W = 16). Every column
    reaches the FP64 true residual and agrees with the single solver."""
    import scipy.sparse as sp

    if case.startswith("band"):
        n = int(case.split("_")[1])
        rp, ci, v = _band_spd(n, 1 if n == 17 else 5)
        A = mf.Matrix.from_csr(n, n, rp, ci, v)
    elif case.startswith("varpoisson3d"):
        A = mf.Matrix.varpoisson3d(3)
    else:
        A = mf.Matrix.poisson2d(10)
    n = A.n
    rp, ci, v = A.csr()
    M = sp.csr_matrix((v, ci, rp), shape=(n, n))
    B = np.random.default_rng(n).uniform(-1, 1, (n, 4))
    X, it, rel, ms = mf.solve_cg_multi(A, B, tol=1e-10, maxiter=2000,
                                       panel=mf.PANEL_FP64 if panel == "fp64" else mf.PANEL_FP32)
    t = mf.Tiles(A)
    for j in range(B.shape[1]):
        b = B[:, j]
        true_rel = np.linalg.norm(b - M @ X[:, j]) / np.linalg.norm(b)
        assert rel[j] <= 1e-10 and true_rel <= 1.01e-10, (case, j, it[j], rel[j], true_rel)
        xs, rs = t.solve_cg(b, tol=1e-10, maxiter=2000)
        assert np.linalg.norm(X[:, j] - xs) / np.linalg.norm(xs) < 1e-8, (case, j)
