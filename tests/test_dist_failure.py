"""A rank that leaves between steps (host-side failure, gloo ranks on CPU):
the surviving rank's next collective -- the per-step norm all-reduce of the
z-slab plan -- ends with an error within the process group's short timeout
instead of waiting for ever."""
import datetime
import os
import socket
import time

import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, port, q):
    import torch
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=2,
                            timeout=datetime.timedelta(seconds=5))
    x = torch.ones(1, dtype=torch.float64)
    dist.all_reduce(x)  # step 1: both ranks
    if rank == 1:
        os._exit(0)  # leaves between steps, no collective in flight
    t0 = time.time()
    try:
        dist.all_reduce(x)  # step 2: the partner is gone
        q.put(("no error", time.time() - t0))
    except Exception as e:  # noqa: BLE001 -- any collective error is the expected outcome
        q.put((type(e).__name__, time.time() - t0))


def test_surviving_rank_gets_an_error_not_a_hang():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    kind, waited = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    assert kind != "no error"
    assert waited < 60
