"""Multi-GPU is replicas only (one process per GPU, no collective on the data
path): the bench's whole-job rate is the units all ranks processed over the
slowest rank's time.  Checked here with world size 2 over gloo on the CPU;
and the reference arm's ranks other than 0 exit without work."""
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


def _rank(rank, world, port, q):
    import torch.distributed as dist
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    import bench
    rate, slowest = bench.replica_rate(100 * (rank + 1), 0.010 * (rank + 1), dist, "cpu")
    q.put((rank, rate, slowest))
    dist.destroy_process_group()


def test_replica_rate_gloo_world_2():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = {}
    for _ in range(2):
        r, rate, slowest = q.get(timeout=120)
        got[r] = (rate, slowest)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # 100 + 200 units over the slower rank's 20 ms, on every rank
    for r in (0, 1):
        assert got[r][1] == pytest.approx(0.020)
        assert got[r][0] == pytest.approx(300 / 0.020)


def test_replica_rate_single_process():
    sys.path.insert(0, ROOT)
    import bench
    assert bench.replica_rate(50, 0.5) == (100.0, 0.5)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference",
                        "--gpus", "2", "--steps", "1", "--warmup", "3"],
                       capture_output=True, text=True, timeout=300, env=env)
    assert r.returncode == 0 and r.stdout.strip() == ""
