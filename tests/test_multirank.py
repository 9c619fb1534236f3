"""The multi-GPU path is replicas only (each rank runs its own simulation,
no collective in the data path); what crosses ranks is the bench's timing:
max over ranks of the device time and the sum of the work.  Checked here
with two gloo ranks on CPU (bench.aggregate_ranks), the same calls the NCCL
run makes."""
import os
import socket

import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

import bench


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    ms = [12.5, 20.0][rank]
    work = [1000.0, 3000.0][rank]
    q.put((rank,) + bench.aggregate_ranks(dist, ms, work, "cpu"))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_take_max_time_and_total_work():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    for _, ms, work in out:
        assert ms == 20.0 and work == 4000.0


def test_single_process_is_identity():
    assert bench.aggregate_ranks(None, 3.0, 7.0, "cpu") == (3.0, 7.0)
