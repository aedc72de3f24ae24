"""The multi-rank host logic of bench.py on CPU with gloo (world size 2):
max-over-ranks timing, the replica aggregate, and failure detection when a
rank leaves before a collective (a short process-group timeout ends the
survivor's barrier with an error instead of a hang)."""
import datetime
import os
import socket
import sys
import time
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parent.parent


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port, timeout_s):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def _max_worker(rank, world, port, out):
    sys.path.insert(0, str(ROOT))
    import bench
    dist = _init(rank, world, port, 30)
    t = bench.max_over_ranks(dist, 1.5 + rank)  # rank 1 is the slow one
    # value = all ranks' work / max rank time (each rank: 10 units)
    out.put((rank, t, bench.replica_value(10.0, world, t)))
    dist.barrier()
    dist.destroy_process_group()


def test_max_over_ranks_and_replica_value_gloo():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_max_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = sorted(q.get(timeout=60) for _ in procs)
    for p in procs:
        p.join(60)
        assert p.exitcode == 0
    assert [g[1] for g in got] == [2.5, 2.5]
    assert all(abs(g[2] - 20.0 / 2.5) < 1e-12 for g in got)


def _leaver(rank, world, port, out):
    dist = _init(rank, world, port, 3)
    dist.barrier()  # both ranks start together
    if rank == 1:
        out.put((rank, "left"))
        out.close()
        out.join_thread()  # the message is written before the process goes
        os._exit(0)  # leaves between steps, with nothing in flight
    t0 = time.monotonic()
    try:
        dist.barrier()
        out.put((rank, "no error"))
    except Exception as e:  # noqa: BLE001 - any collective error is the detection
        out.put((rank, f"detected after {time.monotonic() - t0:.1f}s: {type(e).__name__}"))
    out.close()
    out.join_thread()
    os._exit(0)


def test_survivor_detects_a_rank_that_left():
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_leaver, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    msgs = dict(q.get(timeout=90) for _ in procs)
    for p in procs:
        p.join(30)
    assert msgs[1] == "left"
    assert msgs[0].startswith("detected"), msgs[0]
