"""The N>1 host path on the CPU, world size 2 over gloo.

The path shards by image and pair with no exchange step, so all that runs
across ranks is the timing: each rank's step time is replaced by the maximum
over ranks (`bench.all_ranks_max`) and the job's rate is all ranks' units
over that time.  The reference arm, launched by torchrun as the bench's own
arm is, runs on rank 0 alone and prints one line; the other ranks exit 0.
"""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    import torch
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    import bench
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    assert bench.dist_setup() == (world, rank, rank)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        local_ms = [10.0 + 5.0 * rank, 3.0 * (world - rank)]
        t = torch.tensor(local_ms, dtype=torch.float64)
        same = bench.all_ranks_max(t, world)
        assert same is t
        units_per_rank = 4
        rate = world * units_per_rank / (float(t[0]) / 1e3)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"max": t.tolist(), "rate": rate}, f)
    finally:
        dist.destroy_process_group()


def test_all_ranks_max_gloo_world2(tmp_path):
    import torch.multiprocessing as mp
    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn")
    got = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for g in got:
        assert g["max"] == [15.0, 6.0]
        assert g["rate"] == pytest.approx(2 * 4 / 0.015)


def test_all_ranks_max_single_process_is_identity():
    import torch
    sys.path.insert(0, ROOT)
    import bench
    t = torch.tensor([1.5, 2.5], dtype=torch.float64)
    assert bench.all_ranks_max(t, 1).tolist() == [1.5, 2.5]


def test_reference_arm_under_torchrun_world2():
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", "2",
           "--master-addr", "127.0.0.1", "--master-port", str(_free_port()), "bench.py", "--gpus", "2",
           "--impl", "reference", "--workload", "detect_640x480", "--steps", "1", "--warmup", "3"]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [ln for ln in out.stdout.splitlines() if ln.strip().startswith("{")]
    assert len(lines) == 1, out.stdout
    d = json.loads(lines[0])
    assert d["impl"] == "reference" and d["n_gpus"] == 2 and d["value"] > 0
