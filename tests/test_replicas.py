"""Multi-process (gloo, world size 2, CPU) test of the replica aggregation the
benchmark uses for N > 1: every rank reconstructs its own scene, and the
whole-job throughput is all ranks' samples over the slowest rank's time."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys
    from pathlib import Path
    sys.path.insert(0, str(Path(__file__).resolve().parents[1]))
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    import datetime
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    from bench import replica_throughput
    # rank r pretends to have processed 1000 * (r + 1) samples per step in (r + 1) seconds
    v = replica_throughput(1000 * (rank + 1), float(rank + 1), steps=2, dist=dist)
    out[rank] = v
    dist.barrier()
    dist.destroy_process_group()


def test_replica_throughput_gloo_world2():
    port = _free_port()
    mgr = mp.get_context("spawn").Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(2, port, out), nprocs=2, join=True, start_method="spawn")
    # (1000 + 2000) samples/step * 2 steps / max(1 s, 2 s)
    assert out[0] == pytest.approx(3000.0)
    assert out[1] == pytest.approx(3000.0)


def test_replica_throughput_single():
    from bench import replica_throughput
    assert replica_throughput(500, 2.0, steps=4) == pytest.approx(1000.0)
