"""The FP64 BiCGSTAB kernel's two-reduction form against the oracle's
BiCGSTAB (the reference recurrence, Mille-feuille_BiCGSTAB_NVIDIA.cu:787-1061,
three reductions an iteration), on the CPU.

The kernel (k_bicgstab<false>) folds rho' = r^.r_new into the t.s, t.t
reduction as r^.s - omega r^.t, updates x, r and p in one pass and reduces
that pass's r.r with the next iteration's r^.v, so its stop test runs one
SpMV later with x already final. `two_reduction_bicgstab` below follows that
control flow step for step in NumPy; the test holds its iteration count to
the +-2 % the GPU tests allow and its solution to the oracle's."""
import numpy as np
import pytest


def two_reduction_bicgstab(A, b, tol, maxiter, fixed=False):
    x = np.zeros_like(b)
    r = b - A @ x
    rh = r.copy()
    p = r.copy()
    rr, rho = r @ r, rh @ r
    bn = np.sqrt(b @ b)
    rel = np.sqrt(rr) / bn
    it, rrp, carry = 0, 0.0, False
    while carry or (it < maxiter and (fixed or rel > tol)):
        v = A @ p
        hv = rh @ v  # reduced together with the carried r.r
        if carry:
            carry = False
            rr = rrp
            rel = np.sqrt(rr) / bn
            if it >= maxiter or (not fixed and rel <= tol):
                break  # x is final; this v goes unused
        alpha = rho / hv
        s = r - alpha * v
        t = A @ s
        ts, tt, hs, ht = t @ s, t @ t, rh @ s, rh @ t  # one reduction
        omega = ts / tt
        rho1 = hs - omega * ht
        beta = (rho1 * alpha) / (rho * omega)
        x = x + alpha * p + omega * s
        r = s - omega * t
        p = r + beta * (p - omega * v)
        rrp = r @ r
        rho = rho1
        it += 1
        carry = True
    return it, x, rel


@pytest.mark.parametrize("N,seed", [(24, 0), (40, 3), (64, 0)])
def test_two_reduction_form_matches_oracle_bicgstab(O, N, seed):
    import scipy.sparse as sp

    s = O.gen_convdiff3d(N, seed=seed)  # (64, 0) is the C2 system
    A = sp.csr_matrix((s.v, s.ci, s.rp), shape=(s.n, s.n))
    it_o, x_o, rel_o = O.OracleTiles(s.n, s.n, s.rp, s.ci, s.v).bicgstab(s.b, 1e-10, 5000)
    it, x, rel = two_reduction_bicgstab(A, s.b, 1e-10, 5000)
    assert rel_o <= 1e-10 and rel <= 1e-10
    assert abs(it - it_o) <= max(2, 0.02 * it_o), (it, it_o)
    assert np.linalg.norm(x - x_o) / np.linalg.norm(x_o) < 1e-8
    assert np.linalg.norm(s.b - A @ x) / np.linalg.norm(s.b) <= 1.5e-10


def test_two_reduction_form_fixed_iterations(O):
    import scipy.sparse as sp

    s = O.gen_convdiff3d(16)
    A = sp.csr_matrix((s.v, s.ci, s.rp), shape=(s.n, s.n))
    for k in (0, 1, 5):
        it, x, _ = two_reduction_bicgstab(A, s.b, 1e-10, k, fixed=True)
        assert it == k
        if k == 0:
            assert not x.any()
