"""CG on up to 16 right-hand sides at once: every column against the
single-right-hand-side solver and the CPU oracle's CG."""
import numpy as np
import pytest


@pytest.mark.gpu
@pytest.mark.parametrize("k", [16, 5])
def test_multi_rhs_columns_match_single_solves(mf, O, k):
    import scipy.sparse as sp

    A = mf.Matrix.varpoisson3d(16)
    n = A.n
    rp, ci, v = A.csr()
    rng = np.random.default_rng(20 + k)
    B = rng.uniform(-1, 1, (n, k))
    B[:, 0] = A.b()
    X, it, rel, ms = mf.solve_cg_multi(A, B, tol=1e-10, maxiter=20000)
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
