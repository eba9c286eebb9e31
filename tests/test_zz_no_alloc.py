"""mf_solve_cg_dev_noalloc (static device scratch, no allocation) against
mf_solve_cg_dev, called through the C ABI. The file name sorts last so the
suite also runs it after every other GPU test.

The no-allocation variant runs the FP64 CG kernel with its vectors in global
memory. mf_solve_cg_dev runs that kernel when asked to keep x and r out of
tensor memory (mf_options.reserved[5] = 1): the two then agree to rounding.
Its default, the tensor-memory kernel, sums r.r in another order, so against
it the iteration count is held to the suite's +-2 %."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

RTOL = 1e-12  # same kernel and reduction order: the solutions agree to rounding


def _solve(mf, fn, t, b, x0, opts):
    import torch

    x = x0.clone()
    res = mf.MfResult()
    rc = fn(t.h, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), 1e-10, 20000, C.byref(opts), C.byref(res))
    torch.cuda.synchronize()
    return rc, x, res.as_dict()


@pytest.mark.parametrize("maker", ["varpoisson3d_24", "spd_random_30000"])
def test_noalloc_matches_cg_dev_twice(mf, maker):
    import torch

    kind, size = maker.rsplit("_", 1)
    A = mf.Matrix.varpoisson3d(int(size)) if kind == "varpoisson3d" else mf.Matrix.spd_random(int(size), 9)
    assert -(-A.n // 16) * 16 <= mf.NOALLOC_MAX_ROWS
    L = mf.lib()
    t = mf.Tiles(A)
    o = mf.options(check_true_residual=1)
    b = torch.tensor(A.b(), device="cuda")
    x0 = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    rc, _, r_tm = _solve(mf, L.mf_solve_cg_dev, t, b, x0, o)  # default: x, r in tensor memory
    assert rc == 0 and r_tm["status"] == 0, r_tm
    o_glob = mf.options(check_true_residual=1)
    o_glob.reserved[5] = 1  # the same kernel as the no-allocation variant
    rc, x_ref, r_ref = _solve(mf, L.mf_solve_cg_dev, t, b, x0, o_glob)
    assert rc == 0 and r_ref["status"] == 0, r_ref
    scale = float(x_ref.abs().max())
    for _ in range(2):  # two calls in a row reuse the same scratch
        rc, x, r = _solve(mf, L.mf_solve_cg_dev_noalloc, t, b, x0, o)
        assert rc == 0 and r["status"] == 0, (rc, r, L.mf_last_error())
        assert r["iterations"] == r_ref["iterations"], (r["iterations"], r_ref["iterations"])
        assert abs(r["iterations"] - r_tm["iterations"]) <= max(2, 0.02 * r_tm["iterations"])
        assert float((x - x_ref).abs().max()) <= RTOL * scale
        assert r["rel_residual_true"] <= 1.1e-10, r
        assert abs(r["rel_residual_rec"] - r_ref["rel_residual_rec"]) <= 1e-9 * r_ref["rel_residual_rec"]


def test_noalloc_takes_no_device_memory(mf):
    import torch

    A = mf.Matrix.varpoisson3d(20)
    L = mf.lib()
    o = mf.options()
    b = torch.tensor(A.b(), device="cuda")
    x0 = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    warm = mf.Tiles(A)
    assert _solve(mf, L.mf_solve_cg_dev_noalloc, warm, b, x0, o)[0] == 0  # per-device set-up
    t = mf.Tiles(A)  # fresh handle: mf_solve_cg_dev would allocate its workspace here
    held0 = t.memory_report()
    x = x0.clone()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(2):
        res = mf.MfResult()
        rc = L.mf_solve_cg_dev_noalloc(t.h, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), 1e-10, 20000,
                                       C.byref(o), C.byref(res))
        assert rc == 0
    torch.cuda.synchronize()
    # the handle grew no workspace or sync buffers (the primary check) ...
    held1 = t.memory_report()
    assert held1["workspace_bytes"] == held0["workspace_bytes"] == 0, (held0, held1)
    assert held1["device_bytes"] == held0["device_bytes"]
    # ... and the device's free memory did not move (secondary: another
    # context on a shared device could change it, hence the tolerance of one
    # 2 MiB allocation granule)
    assert abs(torch.cuda.mem_get_info()[0] - free0) < (2 << 20)


def test_noalloc_rejects_oversize(mf):
    import torch

    A = mf.Matrix.poisson2d(400)  # 160000 rows > the static limit
    assert A.n > mf.NOALLOC_MAX_ROWS
    t = mf.Tiles(A)
    b = torch.ones(A.n, dtype=torch.float64, device="cuda")
    x = torch.zeros(A.n, dtype=torch.float64, device="cuda")
    res = mf.MfResult()
    rc = mf.lib().mf_solve_cg_dev_noalloc(t.h, C.c_void_p(b.data_ptr()), C.c_void_p(x.data_ptr()), 1e-10, 100,
                                          C.byref(t.opts), C.byref(res))
    assert rc == mf.MF_ERR_ARG
    assert b"static scratch limit" in mf.lib().mf_last_error()
    assert float(x.abs().max()) == 0.0
