"""The cuSPARSE + cuBLAS baseline that bench.py times beside libmf
(baseline/cusparse) solves the same systems: it reaches the tolerance with
iteration counts close to libmf's FP64 solvers, so the timing comparison
compares like with like."""
import ctypes as C
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _lib():
    path = os.path.join(ROOT, "baseline", "cusparse", "libcusp.so")
    assert os.path.exists(path), "baseline/cusparse not built (run __graft_entry__.build())"
    L = C.CDLL(path)
    for f in ("cusp_cg", "cusp_bicgstab"):
        getattr(L, f).argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                  C.c_double, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_double),
                                  C.POINTER(C.c_double)]
    return L


def _solve(L, fn, A, b, tol, maxiter):
    rp, ci, v = A.csr()
    rp, ci = np.ascontiguousarray(rp, np.int32), np.ascontiguousarray(ci, np.int32)
    v, b = np.ascontiguousarray(v, np.float64), np.ascontiguousarray(b, np.float64)
    x = np.zeros(A.n)
    it, ms, rel = C.c_int(), C.c_double(), C.c_double()
    rc = getattr(L, fn)(A.n, len(v), rp.ctypes.data, ci.ctypes.data, v.ctypes.data, b.ctypes.data, x.ctypes.data,
                        tol, maxiter, C.byref(it), C.byref(ms), C.byref(rel))
    assert rc == 0
    return x, it.value, rel.value


@pytest.mark.parametrize("maker,solver", [("poisson2d_64", "cg"), ("varpoisson3d_24", "cg"),
                                          ("convdiff3d_16", "bicgstab")])
def test_baseline_matches_libmf(mf, maker, solver):
    kind, size = maker.rsplit("_", 1)
    A = getattr(mf.Matrix, kind)(int(size))
    b = A.b()
    L = _lib()
    xc, itc, relc = _solve(L, "cusp_cg" if solver == "cg" else "cusp_bicgstab", A, b, 1e-10, 20000)
    t = mf.Tiles(A)
    x, res = (t.solve_cg if solver == "cg" else t.solve_bicgstab)(b, tol=1e-10, maxiter=20000)
    assert res["status"] == 0 and relc <= 1e-10, (res, relc)
    # the same recurrences in a different summation order
    assert abs(itc - res["iterations"]) <= max(3, 0.03 * res["iterations"]), (itc, res["iterations"])
    rp, ci, v = A.csr()
    r = b - np.array([v[rp[i]:rp[i + 1]] @ xc[ci[rp[i]:rp[i + 1]]] for i in range(A.n)])
    assert np.linalg.norm(r) / np.linalg.norm(b) <= 2e-10
    assert np.linalg.norm(xc - x) <= 1e-6 * np.linalg.norm(x)
