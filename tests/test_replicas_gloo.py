"""Multi-GPU form of the bench: independent replicas, one process per GPU,
whose only collective is the max over ranks of the timed region.  Tested
here with world_size 2 on the gloo backend (CPU): the job value is
world * units / slowest time on every rank, the reference arm prints on
rank 0 only, and a rank that dies makes the others' collective end with an
error instead of hanging."""
import datetime
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import pytest
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _init(rank, world, port):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=20))
    return dist


def _replica_worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    dist = _init(rank, world, port)
    local_ms = [120.0, 200.0][rank]           # rank 1 is the slow one
    m = bench.max_over_ranks(local_ms, dist, device="cpu")
    v = bench.replica_value(world, 1e6, m)
    out.put((rank, m, v))
    dist.destroy_process_group()


def test_max_over_ranks_and_value_gloo():
    world, port = 2, _free_port()
    q = mp.get_context("spawn").SimpleQueue()
    mp.start_processes(_replica_worker, args=(world, port, q), nprocs=world, start_method="spawn", join=True)
    got = sorted(q.get() for _ in range(world))
    for rank, m, v in got:
        assert m == 200.0
        assert v == pytest.approx(world * 1e6 / 0.2 / 1e6)


def _dead_rank_worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import bench
    if rank == 1:
        _init(rank, world, port)
        os._exit(0)                           # leaves between steps, never joins the collective
    try:
        # the dead rank may already be gone while this rank still sets up its
        # connections: an error there ends the collective just the same
        dist = _init(rank, world, port)
        bench.max_over_ranks(1.0, dist, device="cpu")
        out.put((rank, "completed"))
    except Exception as e:                    # noqa: BLE001
        out.put((rank, type(e).__name__))


def test_dead_rank_ends_collective_with_error():
    world, port = 2, _free_port()
    q = mp.get_context("spawn").SimpleQueue()
    ctx = mp.start_processes(_dead_rank_worker, args=(world, port, q), nprocs=world, start_method="spawn",
                             join=False)
    while not ctx.join(timeout=60):
        pass
    rank, what = q.get()
    assert rank == 0 and what != "completed"


def test_reference_arm_prints_on_rank_zero_only(monkeypatch):
    sys.path.insert(0, ROOT)
    import bench
    monkeypatch.setenv("RANK", "1")
    monkeypatch.setattr(sys, "argv", ["bench.py", "--impl", "reference", "--gpus", "2", "--steps", "1",
                                      "--warmup", "0"])
    args = bench.parse()
    buf = io.StringIO()
    with redirect_stdout(buf):
        bench.run_reference(args)
    assert buf.getvalue() == ""
