"""The multi-GPU host logic (independent replicas, max-over-ranks timing)
on two gloo ranks on the CPU, and the reference arm's behaviour on ranks
other than 0."""
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank: int, world: int, port: int, out_dir: str) -> None:
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    from gelios_2d_b200.replicas import max_over_ranks, whole_job_rate

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        # rank r took (r + 1) * 10 ms for 1000 units
        t = max_over_ranks((rank + 1) * 0.010, dist, "cpu")
        rate = whole_job_rate(1000, world, t)
        dist.barrier()
        with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
            f.write(f"{t} {rate}\n")
    finally:
        dist.destroy_process_group()


def test_max_over_ranks_two_gloo_ranks(tmp_path):
    import torch.multiprocessing as mp

    world = 2
    mp.start_processes(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, start_method="spawn",
                       join=True)
    for r in range(world):
        t, rate = map(float, (tmp_path / f"rank{r}.txt").read_text().split())
        assert t == pytest.approx(0.020)  # every rank sees the slowest rank's time
        assert rate == pytest.approx(2 * 1000 / 0.020)


def test_single_process_needs_no_group():
    from gelios_2d_b200.replicas import max_over_ranks, whole_job_rate

    assert max_over_ranks(1.5) == 1.5
    assert whole_job_rate(10, 1, 2.0) == 5.0
    with pytest.raises(ValueError):
        whole_job_rate(10, 1, 0.0)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
