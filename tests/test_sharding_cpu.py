"""History sharding over ranks: the split and the int64 tally sum.

Two gloo ranks on the CPU each transport their slice of the histories (with
the oracle standing in for the CUDA transport of a GPU rank) and sum the
tallies with one all-reduce; the result must equal a single-process run bit
for bit, as it does for the GPU path under NCCL."""
import os
import socket

import numpy as np
import pytest

from gegs_b200.sharding import shard


def test_shard_covers_range_disjoint_and_balanced():
    for h0, h1, world in [(0, 10, 3), (5, 5, 4), (7, 9, 4), (0, 1_000_003, 8), (1 << 40, (1 << 40) + 17, 2)]:
        parts = [shard(h0, h1, r, world) for r in range(world)]
        assert parts[0][0] == h0 and parts[-1][1] == h1
        for (a, b), (c, d) in zip(parts, parts[1:]):
            assert b == c and a <= b
        sizes = [b - a for a, b in parts]
        assert max(sizes) - min(sizes) <= 1


def test_shard_rejects_bad_arguments():
    with pytest.raises(ValueError):
        shard(0, 10, 2, 2)
    with pytest.raises(ValueError):
        shard(10, 0, 0, 1)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, out_path, histories):
    import datetime

    import torch
    import torch.distributed as dist

    from gegs_b200 import workloads as W
    from gegs_b200.sharding import allreduce_tally_
    from oracle import oracle as O
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        job = W.config2(histories=histories, nphsp=2000, n=24)
        a, b = shard(0, histories, rank, world)
        tally, _ = O.run(job.physics, job.scene(), a, b, threads=1)
        t = torch.from_numpy(np.ascontiguousarray(tally, np.int64))
        allreduce_tally_(t)
        if rank == 0:
            np.save(out_path, t.numpy())
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_sum_to_the_single_process_tally(tmp_path, oracle):
    import torch.multiprocessing as mp

    from gegs_b200 import workloads as W
    histories = 1500
    out = str(tmp_path / "tally.npy")
    mp.start_processes(_rank_main, args=(2, _free_port(), out, histories), nprocs=2, join=True,
                       start_method="spawn")
    summed = np.load(out)
    job = W.config2(histories=histories, nphsp=2000, n=24)
    ref, _ = oracle.run(job.physics, job.scene(), 0, histories, threads=1)
    assert summed.sum() > 0
    np.testing.assert_array_equal(summed, ref)
