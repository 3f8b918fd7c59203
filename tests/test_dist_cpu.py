"""The replica path of bench.py on two CPU ranks (gloo over 127.0.0.1): the rendezvous from torchrun's
environment variables, the barrier, the maximum over ranks of each rank's device time, and the whole job's
throughput from it. Replicas exchange nothing else (every rank renders its own frames)."""

import os
import socket
import sys

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out_dir):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    if REPO not in sys.path:
        sys.path.insert(0, REPO)
    import bench

    r, local, w, pg, dev = bench.dist_init(world, backend="gloo")
    assert (r, local, w, dev) == (rank, rank, world, "cpu") and pg is not None
    steps = 5
    device_ms = 10.0 * (rank + 1)  # the ranks' timed device times differ; the job takes the slowest
    bench.barrier(pg, dev)
    slowest = bench.reduce_max(pg, dev, device_ms)
    value = bench.replica_throughput(w, steps, slowest)
    bench.barrier(pg, dev)
    with open(os.path.join(out_dir, f"rank{rank}.txt"), "w") as f:
        f.write(f"{slowest} {value}")
    pg.destroy_process_group()


def test_replicas_on_two_cpu_ranks(tmp_path):
    import torch.multiprocessing as mp

    world, port = 2, _free_port()
    mp.start_processes(_rank, args=(world, port, str(tmp_path)), nprocs=world, start_method="spawn", join=True)
    for rank in range(world):
        slowest, value = (float(v) for v in (tmp_path / f"rank{rank}.txt").read_text().split())
        assert slowest == 10.0 * world
        assert value == pytest.approx(world * 5 / (slowest / 1000.0))


def test_single_process_needs_no_group():
    if REPO not in sys.path:
        sys.path.insert(0, REPO)
    import bench

    for k in ("RANK", "LOCAL_RANK", "WORLD_SIZE"):
        os.environ.pop(k, None)
    rank, local, world, pg, dev = bench.dist_init(1, backend="gloo")
    assert (rank, world, pg) == (0, 1, None)
    assert bench.reduce_max(pg, dev, 3.5) == 3.5
    bench.barrier(pg, dev)
    assert bench.replica_throughput(1, 10, 50.0) == pytest.approx(200.0)
