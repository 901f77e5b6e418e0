"""The N > 1 path runs independent replicas: rank plumbing (barrier,
max-over-ranks timing, per-rank seeds, rank-0 output) over gloo, world size 2,
on CPU."""
import os
import socket
import sys

import pytest
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    sys.path.insert(0, ROOT)
    from quickcbc_b200.replicas import Replicas
    rep = Replicas()
    rep.barrier()
    t = rep.max_over_ranks(10.0 + 5.0 * rank)          # rank 1 is the slower replica
    total = rep.sum_over_ranks(2048)
    out.put((rank, rep.is_root, rep.seed_offset(), t, total))
    rep.close()


def test_two_replicas_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [r[1] for r in res] == [True, False]
    assert [r[2] for r in res] == [0, 1], "each replica draws its own parameter sets"
    assert all(r[3] == 15.0 for r in res), "timing is the max over ranks"
    assert all(r[4] == 4096 for r in res)


def test_single_process_needs_no_backend():
    from quickcbc_b200.replicas import Replicas
    for k in ("RANK", "WORLD_SIZE"):
        os.environ.pop(k, None)
    rep = Replicas()
    assert rep.world == 1 and rep.is_root and rep.max_over_ranks(3.0) == 3.0
