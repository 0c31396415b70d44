"""The N > 1 path of bench.py on CPU: independent replicas, whole-job value summed
over ranks and timed by the slowest rank (two gloo ranks, rendezvous on 127.0.0.1)."""
import os
import socket
import subprocess
import sys

import pytest
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
    # rank r timed (r + 1) * 10 ms for 5 steps and an e2e step of (r + 1) * 2 ms
    res = bench.replica_totals(dist, world, 1_000_000, 5, 10.0 * (rank + 1), 0.002 * (rank + 1), "cpu")
    out[rank] = res
    dist.destroy_process_group()


def test_replica_totals_take_the_slowest_rank():
    world = 2
    port = _free_port()
    out = mp.Manager().dict()
    mp.spawn(_rank, args=(world, port, out), nprocs=world, join=True)
    for r in range(world):
        value, e2e, t_ms, e2e_s = out[r]
        assert t_ms == 20.0 and e2e_s == pytest.approx(0.004)
        assert value == pytest.approx(world * 1e6 * 5 / 0.020 / 1e9)
        assert e2e == pytest.approx(world * 1e6 / 0.004 / 1e9)


def test_reference_arm_other_ranks_exit_without_work():
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--gpus", "2"],
                       env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0
    assert r.stdout.strip() == ""
