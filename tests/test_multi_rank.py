"""The multi-rank path on CPU: two gloo ranks take the steps bench.py takes
under torchrun (the batch workload's longest-processing-time split, the
barrier, the max over ranks of the step time), the split itself is a
balanced partition that every rank computes identically, and the CPU
reference arm runs under torchrun with two ranks."""
import json
import multiprocessing as mp
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_split_is_balanced_partition(mf, world):
    sizes = mf.batch_sizes(512, 1000, 200000, 2)
    parts = mf.split_systems(sizes, world)
    assert len(parts) == world
    flat = sorted(i for p in parts for i in p)
    assert flat == list(range(len(sizes)))
    assert all(p == sorted(p) for p in parts)
    loads = [float(np.sum(sizes[p])) for p in parts]
    # LPT: the spread of the loads is at most one system
    assert max(loads) - min(loads) <= float(sizes.max())
    assert parts == mf.split_systems(sizes, world)


def test_split_edge_cases(mf):
    assert mf.split_systems([], 2) == [[], []]
    assert mf.split_systems([5], 3) == [[0], [], []]
    # ties go to the lower index and the lower rank
    assert mf.split_systems([4, 4, 4, 4], 2) == [[0, 2], [1, 3]]
    with pytest.raises(ValueError):
        mf.split_systems([1], 0)


def test_indexed_generation_matches_whole_batch(mf):
    sizes = [1000, 1300, 900, 1700]
    whole = mf.generate_spd_batch(sizes, seed=2)
    sub = mf.generate_spd_batch([sizes[3], sizes[1]], seed=2, index=[3, 1])
    for a, i in zip(sub, [3, 1]):
        ra, ca, va = a.csr()
        rb, cb, vb = whole[i].csr()
        assert np.array_equal(ra, rb) and np.array_equal(ca, cb) and np.array_equal(va, vb)
    with pytest.raises(ValueError):
        mf.generate_spd_batch([1000], index=[0, 1])


def test_two_gloo_ranks(mf, tmp_path):
    import _dist_worker

    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    procs = [ctx.Process(target=_dist_worker.run, args=(r, world, port, str(tmp_path))) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    for p in procs:
        if p.is_alive():
            p.kill()
            p.join()
    assert [p.exitcode for p in procs] == [0, 0]
    outs = [json.load(open(os.path.join(tmp_path, f"rank{r}.json"))) for r in range(world)]
    sizes = np.array(outs[0]["sizes"])
    # both ranks hold the same split, and it is the single-process split
    assert outs[0]["parts"] == outs[1]["parts"] == mf.split_systems(sizes, world)
    for r in range(world):
        assert outs[r]["parts"][r] == mf.split_systems(sizes, world)[r]
        assert outs[r]["max"] == 3.0
    # the ranks' systems together are the single-process batch
    small = [1000, 1300, 900, 1700, 1100]
    whole = mf.generate_spd_batch(small, seed=2)
    seen = {}
    for o in outs:
        for i, (nnz, s) in zip(o["small_part"], o["small_sums"]):
            seen[i] = (nnz, s)
    assert sorted(seen) == list(range(len(small)))
    for i, m in enumerate(whole):
        assert seen[i] == (int(m.info()[2]), float(m.csr()[2].sum()))


def test_reference_arm_under_torchrun_two_ranks():
    """`bench.py --impl reference` launched as the scaling run launches it:
    rank 0 alone prints one JSON line, rank 1 exits 0 without work, and the
    CPU baseline uses every core the process may run on although torchrun
    sets OMP_NUM_THREADS=1 (a 24^3 grid keeps the test quick)."""
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), os.path.join(root, "bench.py"),
           "--impl", "reference", "--gpus", "2", "--steps", "1", "--warmup", "1", "--grid", "24"]
    p = subprocess.run(cmd, cwd=root, capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = [ln for ln in p.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1, p.stdout
    r = json.loads(lines[0])
    assert r["impl"] == "reference" and r["n_gpus"] == 2 and r["value"] > 0
    assert r["cpu_baseline"]["cores"] == len(os.sched_getaffinity(0))
    assert r["e2e"]["h2d_bytes_per_step"] == 0 and r["e2e"]["value"] == r["value"]
