"""The N > 1 path of bench.py on the CPU: two `gloo` ranks run the replica
plumbing (`bench.Replicas`) that the GPU arm runs over NCCL, and the
reference arm's non-zero ranks exit without work or output."""
import json
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench
    group = bench.Replicas("gloo", device="cpu", timeout_s=60)
    group.barrier()
    # this rank's own step time: rank r is (r + 1) ms
    step_ms = group.max((rank + 1) * 1.0)
    # 3 units per rank in 2 ms (rank 1, the slower) -> 2 * 3 / 0.002
    rate = group.rate(3.0, (rank + 1) * 1e-3)
    group.close()
    with open(os.path.join(out_dir, f"r{rank}.json"), "w") as f:
        json.dump({"step_ms": step_ms, "rate": rate, "world": group.world}, f)


def test_replicas_take_the_slowest_rank(tmp_path):
    import torch.multiprocessing as mp
    world, port = 2, free_port()
    mp.start_processes(_rank, args=(world, port, str(tmp_path)), nprocs=world,
                       start_method="spawn", join=True)
    for r in range(world):
        got = json.loads((tmp_path / f"r{r}.json").read_text())
        assert got["world"] == world
        assert got["step_ms"] == 2.0
        assert got["rate"] == pytest.approx(2 * 3.0 / 2e-3)


def test_single_process_needs_no_group(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    monkeypatch.delenv("RANK", raising=False)
    g = bench.Replicas("gloo", device="cpu")
    assert (g.world, g.rank) == (1, 0)
    assert g.max(1.5) == 1.5 and g.rate(4.0, 2.0) == 2.0
    g.close()


def test_reference_arm_other_ranks_exit_quietly():
    env = {**os.environ, "RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "3", "--warmup", "3"],
                       capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "", r.stdout + r.stderr
