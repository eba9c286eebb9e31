"""One rank of the world-size-2 CPU test (gloo): runs the multi-rank steps
bench.py takes under torchrun and writes what it saw to a JSON file."""
import datetime
import importlib
import json
import os
import sys


def run(rank, world, port, out_dir):
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import torch.distributed as dist

    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        import bench

        mf = importlib.import_module("mille-feillue_b200")
        out = {"rank": rank}
        # the batch workload's split: every rank computes it alone
        sizes = mf.batch_sizes(512, 1000, 200000, 2)
        mine = mf.split_systems(sizes, world)[rank]
        gathered = [None] * world
        dist.all_gather_object(gathered, mine)
        out["parts"] = gathered
        out["sizes"] = [int(s) for s in sizes]
        # a rank's systems are the single-process batch's systems
        small = [1000, 1300, 900, 1700, 1100]
        part = mf.split_systems(small, world)[rank]
        mats = mf.generate_spd_batch([small[i] for i in part], seed=2, index=part)
        out["small_part"] = part
        out["small_sums"] = [[int(m.info()[2]), float(m.csr()[2].sum())] for m in mats]
        # timing: barrier, then the max over ranks of a per-rank value
        bench._barrier(dist)
        out["max"] = bench._max_over_ranks(dist, 1.5 * (rank + 1))
        bench._barrier(dist)
    finally:
        dist.destroy_process_group()
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump(out, f)
