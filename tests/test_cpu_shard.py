"""Sharding a batch over ranks (pysift_b200/shard.py) on the CPU: the
longest-processing-time dealer, and the gather of variable-length results
over two gloo ranks (the collective the GPU path runs over NCCL)."""
import os
import socket
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_lpt_assign_covers_every_unit_once_and_balances():
    from pysift_b200 import shard
    rng = np.random.default_rng(0)
    costs = rng.integers(1, 1000, size=97).astype(float)
    for n in (1, 2, 3, 8):
        share = shard.lpt_assign(costs, n)
        assert len(share) == n
        flat = sorted(i for s in share for i in s)
        assert flat == list(range(len(costs)))
        assert all(s == sorted(s) for s in share)
        loads = [costs[s].sum() for s in share]
        # Graham's bound for LPT: within 4/3 of the optimum, which is at least total / n
        assert max(loads) <= 4.0 / 3.0 * max(costs.sum() / n, costs.max()) + 1e-9
        assert shard.lpt_assign(costs, n) == share  # deterministic


def test_lpt_assign_small_cases():
    from pysift_b200 import shard
    assert shard.lpt_assign([5, 4, 3, 3, 3], 2) == [[0, 3], [1, 2, 4]]
    assert shard.lpt_assign([1, 1], 3) == [[0], [1], []]
    assert shard.lpt_assign([], 2) == [[], []]
    with pytest.raises(ValueError):
        shard.lpt_assign([1], 0)


def test_batch_costs_follow_pixel_counts():
    from pysift_b200 import shard, synthetic
    sizes = synthetic.pair_sizes(32, 0)
    share = shard.lpt_assign([shard.pair_cost(s, s) for s in sizes], 4)
    loads = [sum(2 * sizes[i][0] * sizes[i][1] for i in s) for s in share]
    assert max(loads) / min(loads) < 1.2


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _gather_main(rank, world, port, out_dir, n_total):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    from pysift_b200 import shard
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        costs = [float((i * 37) % 11 + 1) for i in range(n_total)]
        share = shard.lpt_assign(costs, world)[rank]
        # unit i has i % 4 rows (unit 0: none) of 5 columns, value 100 i + row
        local = {i: torch.arange(i % 4, dtype=torch.float32)[:, None].repeat(1, 5) + 100.0 * i for i in share}
        got = shard.gather_rows(local, n_total)
        np.save(os.path.join(out_dir, f"rank{rank}.npy"),
                np.array([g.numpy() for g in got], dtype=object), allow_pickle=True)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_total", [7, 1])
def test_gather_rows_gloo_world2(tmp_path, n_total):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_gather_main, args=(world, _free_port(), str(tmp_path), n_total), nprocs=world,
                       start_method="spawn")
    for r in range(world):
        got = np.load(tmp_path / f"rank{r}.npy", allow_pickle=True)
        assert len(got) == n_total
        for i, g in enumerate(got):
            want = np.arange(i % 4, dtype=np.float32)[:, None].repeat(5, 1) + 100.0 * i
            assert g.shape == (i % 4, 5) and np.array_equal(g, want)
