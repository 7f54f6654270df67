"""The multi-GPU path of bench.py on CPU: world-size-2 process groups over
gloo.  Ranks are replicas (rays are independent, no data exchange); the step
time is the maximum over ranks and the job throughput counts every rank's
rays; under torchrun the reference arm runs on rank 0 alone."""
import os
import socket
import subprocess
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import torch
    import torch.distributed as dist

    sys.path.insert(0, str(ROOT))
    import bench

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    local_ms = [0.40, 0.55][rank]
    ms = bench.max_over_ranks(local_ms, world, torch.device("cpu"))
    out[rank] = (ms, bench.job_mrays_per_s(world, 2_073_600, ms))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_job_throughput():
    world = 2
    out = mp.Manager().dict()
    mp.start_processes(_rank_main, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    assert out[0] == out[1]
    ms, value = out[0]
    assert ms == pytest.approx(0.55)
    assert value == pytest.approx(2 * 2_073_600 / 0.55e-3 / 1e6)


def test_reference_arm_other_ranks_exit_quietly():
    """`bench.py --impl reference` under torchrun: ranks other than 0 do no
    work and print nothing."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], env=env, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
