"""Numerics of the multi-right-hand-side panel product's precision (CPU).

The block-CG workload's specification names a BF16 tile x panel product
on tensor cores. These tests restate that product on the CPU for one column
(q = fl32(bf16(A) bf16(p)): BF16 off-diagonal entries and directions, the
diagonal in FP32 as in the mixed layouts, exact products, FP32 result),
inside the CG the panel kernel runs (FP64 x, r, dots and scalars, r replaced
by b - A x every 50 iterations, convergence on the true residual), on the
24^3 variable-coefficient Poisson of the oracle's generator:

* BF16 tiles rounded entry by entry make the operator indefinite: the solve
  does not reach 1e-10 (it diverges);
* with the row-sum-preserving compensation of the mixed layouts (the
  diagonal absorbs the row's rounding) the BF16 product converges, with
  more iterations than FP64;
* FP32 search directions with the exact matrix (what MF_PANEL_FP32 runs)
  stay within a few percent of FP64.
"""
import numpy as np
import pytest
import scipy.sparse as sp

import _oracle as O

TOL = 1e-10


def bf16(a):
    """Round to the nearest BF16 (ties to even), returned as float64."""
    u = np.asarray(a, np.float32).view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def f32(a):
    return np.asarray(a, np.float32).astype(np.float64)


@pytest.fixture(scope="module")
def system():
    m = O.gen_varpoisson3d(24)
    rp, ci, v = m.csr()
    n = m.n
    A = sp.csr_matrix((v, ci, rp), shape=(n, n))
    rows = np.repeat(np.arange(n), np.diff(rp))
    b = np.random.default_rng(0).uniform(-1, 1, n)
    return A, rp, ci, v, rows, b


def panel_operator(system, kind):
    A, rp, ci, v, rows, _ = system
    n = A.shape[0]
    if kind == "fp64" or kind == "fp32dir":
        return A
    off = ci != rows
    vl = v.copy()
    vl[off] = bf16(v[off])
    dg = ~off
    if kind == "bf16_comp":  # the diagonal (FP32) absorbs the row's rounding
        d = np.bincount(rows[off], weights=vl[off] - v[off], minlength=n)
        vl[dg] = f32(v[dg] - d[rows[dg]])
    else:
        vl[dg] = f32(v[dg])
    return sp.csr_matrix((vl, ci, rp), shape=(n, n))


def cg(system, kind, maxiter):
    A, _, _, _, _, b = system
    Ap = panel_operator(system, kind)
    rnd = {"fp64": lambda z: z, "fp32dir": f32}.get(kind, bf16)
    x = np.zeros_like(b)
    r = b.copy()
    p = np.array(rnd(r))  # a copy: r is updated in place
    rr, bb = r @ r, b @ b
    for it in range(1, maxiter + 1):
        q = Ap @ p if kind == "fp64" else f32(Ap @ p)
        a = rr / (p @ q)
        if not np.isfinite(a) or a <= 0:
            return -1
        x += a * p
        r -= a * q
        rn = r @ r
        if it % 50 == 0 or np.sqrt(rn / bb) <= TOL:
            r = b - A @ x
            rn = r @ r
            if np.sqrt(rn / bb) <= TOL:
                return it
        if not np.isfinite(rn):
            return -1
        p = rnd(r + (rn / rr) * p)
        rr = rn
    return -1


def test_bf16_panel_needs_row_sum_compensation(system):
    it64 = cg(system, "fp64", 20000)
    assert it64 > 0
    assert cg(system, "bf16", 3 * it64) == -1  # uncompensated BF16 tiles: no convergence
    itc = cg(system, "bf16_comp", 3 * it64)
    assert 0 < itc <= 1.5 * it64, (itc, it64)
    it32 = cg(system, "fp32dir", 3 * it64)
    assert 0 < it32 <= 1.06 * it64, (it32, it64)
