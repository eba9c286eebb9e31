"""The slab planner runs on the GPU (k_plan). With the planner check on,
every layout built is planned again by the host planner (the same greedy
rules) and each plan, segment and run is compared: FP64 and mixed layouts,
staged, gather and oversize slabs, FP32-x and FP64-x windows, small stages
and the C3 matrix itself."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dense_rows(n, seed):
    rng = np.random.default_rng(seed)
    rp, ci, va = [0], [], []
    for r in range(n):
        cols = set(rng.integers(0, n, size=4).tolist()) | {r}
        if r in (5, 6, 7, n // 2):
            cols |= set(range(n))
        cols = sorted(cols)
        ci += cols
        va += rng.standard_normal(len(cols)).tolist()
        rp.append(len(ci))
    return n, np.array(rp, np.int32), np.array(ci, np.int32), np.array(va)


def test_gpu_planner_matches_host_planner(mf):
    mf.check_planner(True)
    try:
        cases = [(mf.Matrix.varpoisson3d(128), {}), (mf.Matrix.varpoisson3d(128), dict(precision_mode=mf.MODE_MIXED_RULE)),
                 (mf.Matrix.poisson2d(256), dict(precision_mode=mf.MODE_MIXED_RULE)),
                 (mf.Matrix.convdiff3d(40), dict(slab_bytes=4096, rb_per_slab=3)),
                 (mf.Matrix.spd_random(30000, 4), dict(precision_mode=mf.MODE_MIXED_RULE)),
                 (mf.Matrix.spd_random(30000, 4), dict(slab_bytes=2048, rb_per_slab=1))]
        for A, kw in cases:
            t = mf.Tiles(A, mf.options(**kw))
            del t
        n, rp, ci, v = _dense_rows(4000, 2)
        for kw in ({}, dict(precision_mode=mf.MODE_FIXED, fixed_precision=mf.PREC_FP16)):
            t = mf.Tiles(csr=(n, n, rp, ci, v), opts=mf.options(**kw))
            del t
        checked, bad = mf.check_planner()
        assert checked >= 10 and bad == 0, (checked, bad)
    finally:
        mf.check_planner(False)
