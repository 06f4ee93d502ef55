"""Multi-rank host logic of bench.py on CPU (gloo, world_size 2): every rank
runs an independent replica, the timed figure is the slowest rank's, and the
whole-job throughput counts every replica. The path itself does not shard, so
there is no data-path collective to test."""
import importlib.util
import json
import os
import pathlib
import subprocess
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parent.parent


def load_bench():
    spec = importlib.util.spec_from_file_location("ow3d_bench", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def _worker(rank, world, port, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        b = load_bench()
        ms = 100.0 + 25.0 * rank
        slow = b.max_over_ranks(ms, world, "cpu")
        dist.barrier()
        with open(out / f"r{rank}.json", "w") as f:
            json.dump({"slow": slow, "seed": b.replica_seed(rank),
                       "value": b.job_throughput(1000, 4, world, slow)}, f)
    finally:
        dist.destroy_process_group()


def test_two_rank_replicas_gloo(tmp_path):
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    mp.start_processes(_worker, args=(2, port, tmp_path), nprocs=2, join=True, start_method="spawn")
    r = [json.loads((tmp_path / f"r{i}.json").read_text()) for i in range(2)]
    assert r[0]["slow"] == r[1]["slow"] == 125.0
    assert r[0]["seed"] != r[1]["seed"]
    # 2 replicas x 1000 DOF x 4 steps in 0.125 s
    assert abs(r[0]["value"] - 2 * 1000 * 4 / 0.125) < 1e-9


def test_single_rank_needs_no_process_group():
    b = load_bench()
    assert b.max_over_ranks(3.5, 1, "cpu") == 3.5
    assert b.job_throughput(10, 2, 1, 1000.0) == 20.0


def test_reference_arm_other_ranks_exit_quietly():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1", "--warmup", "0"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == ""
