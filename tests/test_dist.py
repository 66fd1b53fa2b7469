"""Host-side multi-rank logic of bench.py with the gloo backend, world size 2."""
import os
import socket

import torch.multiprocessing as mp

from scft_string_b200 import dist as D


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    r, w, lr = D.env()
    D.init("gloo", timeout_s=60)
    D.barrier(w)
    ms = 100.0 * (rank + 1)          # rank 1 is the slower one
    mx = D.max_over_ranks(ms, w)
    q.put((r, lr, mx, D.job_rate(5, w, mx)))
    D.finalize(w)


def test_two_rank_max_and_rate():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    for p in ps:
        p.join(120)
        assert p.exitcode == 0
    out = sorted(q.get() for _ in range(2))
    for r, (rank, lr, mx, rate) in enumerate(out):
        assert rank == r and lr == r
        assert mx == 200.0
        assert abs(rate - 2 * 5 / 0.2) < 1e-9


def test_single_rank_defaults():
    assert D.max_over_ranks(3.5, 1) == 3.5
    assert D.job_rate(10, 1, 1000.0) == 10.0
