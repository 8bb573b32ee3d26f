"""The N > 1 path without GPUs: two gloo ranks on CPU shard a batch, reduce a
per-rank time to its maximum and gather the slices back (accelerint_b200/shard.py)."""
import os
import socket

import numpy as np
import pytest

from accelerint_b200.shard import shard_range


def test_shard_range_partitions():
    for num in (0, 1, 7, 1001, 65536):
        for world in (1, 2, 3, 8):
            spans = [shard_range(num, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == num
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [b - a for a, b in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, num, out_dir):
    import torch.distributed as dist
    from datetime import timedelta
    from accelerint_b200.shard import gather_columns, max_over_ranks, shard_columns
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        rng = np.random.default_rng(5)
        y = rng.standard_normal((3, num))
        var = rng.standard_normal(num)
        yl, vl = shard_columns(y, var, rank, world)
        # stand-in for an integration step: every column handled independently
        yl = 2.0 * yl + vl[None, :]
        t_max = max_over_ranks(10.0 + rank)
        full = gather_columns(yl, num)
        np.save(os.path.join(out_dir, f"r{rank}.npy"), full)
        with open(os.path.join(out_dir, f"t{rank}.txt"), "w") as f:
            f.write(repr(t_max))
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_shard_reduce_gather(tmp_path):
    import torch.multiprocessing as mp
    num, world = 1001, 2
    mp.spawn(_worker, args=(world, _free_port(), num, str(tmp_path)), nprocs=world, join=True)
    rng = np.random.default_rng(5)
    y = rng.standard_normal((3, num))
    var = rng.standard_normal(num)
    expect = 2.0 * y + var[None, :]
    for r in range(world):
        assert np.array_equal(np.load(tmp_path / f"r{r}.npy"), expect)
        assert float(open(tmp_path / f"t{r}.txt").read()) == 11.0
