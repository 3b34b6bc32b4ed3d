"""The multi-process path of the hot paths on CPU: two gloo ranks shard a set of
trajectories, each produces its share of a per-trajectory result, and the
gathered result and the max-over-ranks timing equal the single-process ones."""
import os
import socket

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from mqct_b200 import replicas


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, n, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        b, e = replicas.shard(n, rank, world)
        # a per-trajectory result (deterministic in the trajectory index)
        rows = np.array([[i, i * i, np.sin(i)] for i in range(b, e)], dtype=np.float64).reshape(-1, 3)
        full = replicas.gather_rows(rows, n, dist)
        t = replicas.max_over_ranks(1.5 + rank, dist)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), full)
        with open(os.path.join(out_dir, f"t{rank}.txt"), "w") as f:
            f.write(repr(t))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n", [7, 8, 1])
def test_shard_gather_and_max_over_two_gloo_ranks(tmp_path, n):
    world = 2
    mp.start_processes(_worker, args=(world, _free_port(), n, str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    ref = np.array([[i, i * i, np.sin(i)] for i in range(n)], dtype=np.float64)
    for r in range(world):
        got = np.load(tmp_path / f"r{r}.npy")
        assert np.array_equal(got, ref)
        assert float(open(tmp_path / f"t{r}.txt").read()) == 2.5


def test_shards_cover_without_overlap():
    for n in (0, 1, 5, 148, 4096):
        for world in (1, 2, 3, 8):
            spans = [replicas.shard(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            assert max(e - b for b, e in spans) - min(e - b for b, e in spans) <= 1
    with pytest.raises(ValueError):
        replicas.shard(4, 2, 2)
