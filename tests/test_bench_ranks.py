"""bench.py's multi-rank plumbing on CPU: two gloo ranks combine their
device times (max) and traversed edges (sum) exactly as the NCCL ranks do on
GPUs, every rank sees the same job figures, and the reference arm runs on
rank 0 only."""
import os
import socket
import subprocess
import sys

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist

    sys.path.insert(0, ROOT)
    import bench

    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    ms = [12.5, 17.25][rank]
    edges = [3_000_000_007, 5_000_000_011][rank]
    out[rank] = bench.combine_ranks(dist, ms, edges, "cpu")
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_combine_time_and_edges():
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.start_processes(_rank, args=(2, port, out), nprocs=2, start_method="spawn", join=True)
        got = dict(out)
    assert got[0] == got[1] == (17.25, 8_000_000_018)


def test_combine_without_a_process_group():
    sys.path.insert(0, ROOT)
    import bench

    assert bench.combine_ranks(None, 3.5, 42, "cpu") == (3.5, 42)


def test_reference_arm_prints_nothing_on_other_ranks():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "0"], capture_output=True, text=True, env=env, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""
