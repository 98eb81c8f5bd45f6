"""The multi-GPU form of bench.py on CPU ranks (gloo, world size 2): each rank
draws its own shard of cells (no cell data crosses ranks), the timing is the
maximum over ranks, and the whole-job rate counts every rank's cells."""
import os
import socket
import sys
from pathlib import Path

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as tmp

REPO = Path(__file__).resolve().parents[1]


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    sys.path.insert(0, str(REPO))
    import datetime

    import bench
    from kpp_b200 import load, workloads
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        mech = load("saprc99")
        wl = workloads.for_mechanism(mech, "saprc99_uniform95", 64, seed=bench.shard_seed(rank))
        cpu = torch.device("cpu")
        ms = 100.0 + 50.0 * rank  # a slower second rank
        ms_max = bench.reduce_max(ms, cpu)
        checksum = torch.tensor([float(wl.var.sum())], dtype=torch.float64)
        all_sums = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
        dist.all_gather(all_sums, checksum)
        rate = bench.whole_job_rate(64, world, 3, ms_max)
        np.save(Path(out_dir) / f"rank{rank}.npy",
                np.array([ms_max, rate] + [float(t.item()) for t in all_sums]))
    finally:
        dist.destroy_process_group()


def test_two_ranks_shard_and_time_like_the_benchmark(tmp_path):
    world = 2
    tmp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    r0, r1 = (np.load(tmp_path / f"rank{r}.npy") for r in range(world))
    assert r0[0] == r1[0] == 150.0            # the slowest rank's time on every rank
    assert r0[1] == r1[1] == 2 * 64 * 3 / 0.150  # every rank's cells over that time
    assert r0[2] != r0[3]                      # the two shards are different cells
    np.testing.assert_array_equal(r0[2:], r1[2:])
