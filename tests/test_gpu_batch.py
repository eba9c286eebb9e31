"""Batched persistent launch: groups of CTAs take systems from a queue and
solve each with group-local reductions; compared with the single-system
solver and the CPU oracle for several group sizes."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("gs", [1, 4, 8, 16])
def test_batch_matches_single_system_solver(mf, O, gs):
    import torch

    sizes = [1000, 1500, 2333, 4000, 777, 16, 5000, 12000, 3000, 9000]
    mats = [mf.Matrix.spd_random(n, 100 + i) for i, n in enumerate(sizes)]
    mats.append(mf.Matrix.poisson2d(40))
    o = mf.options()
    o.reserved[4] = gs
    B = mf.Batch(mats, o, with_baseline=True)
    assert B.info()["grid"] == (148 // gs) * gs or B.info()["grid"] % gs == 0
    b = np.concatenate([m.b() for m in mats])
    bd = torch.tensor(b, device="cuda")
    xd = torch.zeros_like(bd)
    ms = B.solve_cg_dev(bd.data_ptr(), xd.data_ptr(), 1e-10, 10000)
    assert ms > 0
    it, st, rel = B.results()
    assert np.all(st == 0) and np.all(rel <= 1e-10)
    x = xd.cpu().numpy()
    # graph replay gives the identical answer
    xd2 = torch.zeros_like(bd)
    B.solve_cg_dev(bd.data_ptr(), xd.data_ptr(), 1e-10, 10000)
    assert np.array_equal(xd.cpu().numpy(), x)
    off = B.offsets
    import scipy.sparse as sp

    for s, m in enumerate(mats):
        rp, ci, v = m.csr()
        n = m.n
        M = sp.csr_matrix((v, ci, rp), shape=(n, n))
        xs = x[off[s]:off[s + 1]]
        assert np.linalg.norm(m.b() - M @ xs) / np.linalg.norm(m.b()) <= 1.5e-10
        o = O.OracleTiles(n, n, rp, ci, v)
        it_o, _, _ = o.cg(m.b(), 1e-10, 10000)
        assert abs(int(it[s]) - it_o) <= max(2, 0.02 * it_o), (s, it[s], it_o)
    # one launch per system
    B.solve_cg_each_dev(bd.data_ptr(), xd2.data_ptr(), 1e-10, 10000)
    it2, st2, rel2 = B.results()
    assert np.all(st2 == 0)
    assert np.max(np.abs(it2 - it)) <= 2
    assert np.linalg.norm(xd2.cpu().numpy() - x) / np.linalg.norm(x) < 1e-8


def test_batch_c4_subset_64_systems(mf, O):
    """64 systems drawn from the 512-system workload itself (every 8th of the
    seeded size list, n log-uniform in [1e3, 2e5], the same per-system seeds),
    about 2.4 M rows: one persistent launch against one launch per system,
    the true residual of every system, and the oracle's iterations on a
    spread of them."""
    import scipy.sparse as sp
    import torch

    sizes = mf.batch_sizes(512, 1000, 200000, 2)
    pick = list(range(0, 512, 8))
    mats = mf.generate_spd_batch([sizes[s] for s in pick], seed=2, index=pick)
    assert sum(m.n for m in mats) > 1_000_000
    B = mf.Batch(mats, mf.options(), with_baseline=True)
    b = np.concatenate([m.b() for m in mats])
    bd = torch.tensor(b, device="cuda")
    xd = torch.zeros_like(bd)
    B.solve_cg_dev(bd.data_ptr(), xd.data_ptr(), 1e-10, 10000)
    it, st, rel = B.results()
    assert np.all(st == 0) and np.all(rel <= 1e-10)
    x = xd.cpu().numpy()
    off = B.offsets
    for s, m in enumerate(mats):
        rp, ci, v = m.csr()
        M = sp.csr_matrix((v, ci, rp), shape=(m.n, m.n))
        assert np.linalg.norm(m.b() - M @ x[off[s]:off[s + 1]]) / np.linalg.norm(m.b()) <= 1.5e-10, s
    order = np.argsort([m.n for m in mats])
    for s in order[:: len(order) // 8]:
        m = mats[s]
        rp, ci, v = m.csr()
        it_o, _, _ = O.OracleTiles(m.n, m.n, rp, ci, v).cg(m.b(), 1e-10, 10000)
        assert abs(int(it[s]) - it_o) <= max(2, 0.02 * it_o), (s, it[s], it_o)
    xe = torch.zeros_like(bd)
    B.solve_cg_each_dev(bd.data_ptr(), xe.data_ptr(), 1e-10, 10000)
    it2, st2, _ = B.results()
    assert np.all(st2 == 0) and np.max(np.abs(it2 - it)) <= 2
    assert np.linalg.norm(xe.cpu().numpy() - x) / np.linalg.norm(x) < 1e-8
