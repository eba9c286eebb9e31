"""Learned precision selector: the GPU forward and backward kernels against
the CPU oracle's MLP, training, the selector fused into the feature pass,
and the magnitude-rule fallback of the solve."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

NW = 4868


def _weights(seed, scale=0.2):
    return (np.random.default_rng(seed).standard_normal(NW) * scale).astype(np.float32)


def _dev(a):
    import torch

    return torch.tensor(a, device="cuda")


def test_forward_matches_oracle(mf, O):
    import ctypes as C
    import torch

    w = _weights(1)
    x = np.random.default_rng(2).standard_normal((1500, 6)).astype(np.float32)
    wd, xd = _dev(w), _dev(x)
    out = torch.zeros((1500, 4), dtype=torch.float32, device="cuda")
    assert mf.lib().mf_mlp_forward_dev(C.c_void_p(wd.data_ptr()), C.c_void_p(xd.data_ptr()), 1500, 0,
                                       C.c_void_p(out.data_ptr())) == 0
    ref = O.mlp_forward(w, x)
    assert np.max(np.abs(out.cpu().numpy() - ref)) <= 1e-5 * max(1.0, np.max(np.abs(ref)))


def test_gradient_matches_oracle(mf, O):
    """Samples span several blocks of the kernel (512 each), so the fixed-order
    sum of the per-block partial gradients is exercised too."""
    import ctypes as C
    import torch

    rng = np.random.default_rng(3)
    w = _weights(4)
    n = 2600
    x = rng.standard_normal((n, 6)).astype(np.float32)
    y = rng.integers(0, 4, n).astype(np.int32)
    g = torch.zeros(NW, dtype=torch.float32, device="cuda")
    loss = C.c_float()
    wd, xd, yd = _dev(w), _dev(x), torch.tensor(y, device="cuda")
    assert mf.lib().mf_mlp_grad_dev(C.c_void_p(wd.data_ptr()), C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()),
                                    n, C.c_void_p(g.data_ptr()), C.byref(loss)) == 0
    g_ref, loss_ref = O.mlp_grad(w, x, y)
    gg = g.cpu().numpy()
    assert abs(loss.value - loss_ref) <= 1e-5 * abs(loss_ref)
    # FP32 sums in different orders: tolerance relative to the gradient's size
    assert np.linalg.norm(gg - g_ref) <= 1e-5 * np.linalg.norm(g_ref)
    assert np.max(np.abs(gg - g_ref)) <= 1e-5 * np.max(np.abs(g_ref))
    # the gradient is deterministic
    g2 = torch.zeros_like(g)
    mf.lib().mf_mlp_grad_dev(C.c_void_p(wd.data_ptr()), C.c_void_p(xd.data_ptr()), C.c_void_p(yd.data_ptr()), n,
                             C.c_void_p(g2.data_ptr()), C.byref(loss))
    assert torch.equal(g, g2)


def test_training_learns_a_rule(mf):
    """Labels from a threshold rule on two features: Adam on the GPU kernels
    fits it to > 97 % training accuracy."""
    import ctypes as C
    import torch

    rng = np.random.default_rng(5)
    n = 20000
    x = rng.uniform(-1, 1, (n, 6)).astype(np.float32)
    y = np.where(x[:, 0] > 0.3, 0, np.where(x[:, 0] > -0.2, 1, np.where(x[:, 3] > 0, 1, 2))).astype(np.int32)
    w = _weights(6, 0.1)
    wd, xd, yd = _dev(w), _dev(x), torch.tensor(y, device="cuda")
    loss = C.c_float()
    assert mf.lib().mf_mlp_train_dev(C.c_void_p(wd.data_ptr()), C.c_void_p(xd.data_ptr()),
                                     C.c_void_p(yd.data_ptr()), n, 1500, 512, C.c_float(3e-3), C.byref(loss)) == 0
    out = torch.zeros((n, 4), dtype=torch.float32, device="cuda")
    mf.lib().mf_mlp_forward_dev(C.c_void_p(wd.data_ptr()), C.c_void_p(xd.data_ptr()), n, 0, C.c_void_p(out.data_ptr()))
    acc = float(np.mean(out.cpu().numpy().argmax(1) == y))
    assert acc > 0.97, (acc, loss.value)


def _select_numpy(logits, f):
    """The selector's class with its hard limits (k_tile_select_mlp)."""
    c = logits.argmax(1)
    c = np.where((c == 3) & (f[:, 1] > 3.6124), 2, c)
    c = np.where((c == 2) & (f[:, 1] > 8.0), 1, c)
    c = np.where(~np.isfinite(f[:, 0]) | (f[:, 0] > 300), 0, c)
    return c


def test_fused_selector_equals_features_plus_forward(mf):
    """The selector fused into the feature pass (BF16 weights) gives the class
    of the separate feature export + BF16 forward."""
    import ctypes as C
    import torch

    A = mf.Matrix.varpoisson3d(12, 1e-2, 1e2, 3)
    t = mf.Tiles(A)
    w = _weights(7, 0.5)
    mf.set_mlp_weights(w)
    try:
        levels = np.array([1.0, 1e-6])
        p = t.select_mlp(levels)
        f = t.features()
        assert np.allclose(f[:, 2], np.log10(A.nnz), atol=1e-5)  # whole-matrix nnz feature
        for l, res in enumerate(levels):
            fl = f.copy()
            fl[:, 5] = np.log10(res)
            out = torch.zeros((len(f), 4), dtype=torch.float32, device="cuda")
            wd, fd = _dev(w), _dev(fl)
            mf.lib().mf_mlp_forward_dev(C.c_void_p(wd.data_ptr()), C.c_void_p(fd.data_ptr()), len(f), 1,
                                        C.c_void_p(out.data_ptr()))
            logits = out.cpu().numpy()
            srt = np.sort(logits, 1)
            clear = (srt[:, 3] - srt[:, 2]) > 1e-4  # near-ties may break either way
            assert np.array_equal(p[l][clear], _select_numpy(logits, fl)[clear])
            assert clear.mean() > 0.99
    finally:
        mf.set_mlp_weights(None)


def test_selector_fallback_to_rule(mf):
    """A selector solve that runs more than 10 % over the reference iteration
    count (mf_options.reserved[6]) is solved again with the rule from the
    same x0, and the result says so. The weights put every tile in FP8 (the
    row-sum-preserving storage keeps even that solve convergent on this
    matrix, so the reference count forces the fallback)."""
    A = mf.Matrix.varpoisson3d(20)
    b = A.b()
    w = np.zeros(NW, np.float32)
    w[4864:4868] = [0.0, 0.0, 0.0, 10.0]  # b3: class FP8 everywhere
    mf.set_mlp_weights(w)
    try:
        t = mf.Tiles(A, mf.options(precision_mode=mf.MODE_MIXED_MLP))
        p, _ = t.precisions()
        assert (p >= mf.PREC_FP16).mean() > 0.5
        o = mf.options(precision_mode=mf.MODE_MIXED_MLP)
        o.reserved[6] = 100  # reference iteration count: the FP8 solve runs over it
        x, res = t.solve_cg(b, tol=1e-10, maxiter=20000, opts=o)
        assert res["selector_fallback"] == 1, res
        assert res["status"] == 0 and res["rel_residual_true"] <= 1e-10, res
    finally:
        mf.set_mlp_weights(None)


def test_packaged_selector_solves(mf):
    """The trained selector shipped with the package reaches the FP64 true
    residual on a held-out matrix of the training family."""
    import os

    if not os.path.exists(mf.MLP_WEIGHTS_PATH):
        pytest.skip("no trained selector weights packaged")
    A = mf.Matrix.varpoisson3d(40, 10 ** -2.5, 10 ** 2.5, 901)
    b = A.b()
    try:
        t = mf.Tiles(A, mf.options(precision_mode=mf.MODE_MIXED_MLP))
        x, res = t.solve_cg(b, tol=1e-10, maxiter=40000)
        assert res["status"] == 0 and res["rel_residual_true"] <= 1e-10, res
    finally:
        mf.set_mlp_weights(None)


@pytest.mark.gpu
def test_packaged_selector_gain_over_rule(mf):
    """What the trained selector gains over the precision rule, measured
    against the FP64 solve, on held-out matrices of the training family (grids and seeds
    outside the training set, contrasts over the training range): iterations,
    SpMV bytes and solve time of the selector's mixed solve against the
    rule's. Both must reach the 1e-10 FP64 true residual and stay within
    1e-6 of the FP64 solution; the selector must not fall back, must not
    lose more than 10 % of the rule's iterations nor add SpMV bytes. The
    measured ratios are printed (on this family the rule already stores
    every tile at the lowest precision that converges, FP16 with FP32
    diagonals, and the selector reproduces it: ratios 1.0)."""
    import os

    if not os.path.exists(mf.MLP_WEIGHTS_PATH):
        pytest.skip("no trained selector weights packaged")
    gains = []
    for grid, lg, seed in ((44, 1.5, 7001), (52, 4.0, 7002), (60, 7.0, 7003)):
        A = mf.Matrix.varpoisson3d(grid, 10 ** (-lg / 2), 10 ** (lg / 2), seed)
        b = A.b()
        x64, r64 = mf.Tiles(A).solve_cg(b, tol=1e-10, maxiter=40000)
        tr = mf.Tiles(A, mf.options(precision_mode=mf.MODE_MIXED_RULE))
        xr, rr = tr.solve_cg(b, tol=1e-10, maxiter=40000)
        o = mf.options(precision_mode=mf.MODE_MIXED_MLP)
        o.reserved[6] = rr["iterations"]
        tm = mf.Tiles(A, o)
        xm, rm = tm.solve_cg(b, tol=1e-10, maxiter=40000, opts=o)
        for x, r in ((xr, rr), (xm, rm)):
            assert r["status"] == 0 and r["rel_residual_true"] <= 1e-10, r
            assert np.linalg.norm(x - x64) / np.linalg.norm(x64) < 1e-6
        assert rm["selector_fallback"] == 0, rm
        assert rm["iterations"] <= 1.1 * rr["iterations"], (rm["iterations"], rr["iterations"])
        assert rm["spmv_bytes_level"][0] <= rr["spmv_bytes_level"][0] * (1 + 1e-9)
        gains.append({"grid": grid, "log10_contrast": lg, "fp64_iters": r64["iterations"],
                      "iters_rule_over_mlp": rr["iterations"] / rm["iterations"],
                      "bytes_rule_over_mlp": rr["spmv_bytes_level"][0] / rm["spmv_bytes_level"][0],
                      "time_rule_over_mlp": rr["time_ms"] / rm["time_ms"]})
    print("selector gain over the rule:", gains)
