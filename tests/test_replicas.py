"""CPU: the multi-process plumbing of bench.py under torchrun (replicas only).

Two ranks on the gloo backend, rendezvous on 127.0.0.1: the timing reduction
takes the maximum over ranks, the barrier releases both ranks, and the
reference arm prints nothing on a rank other than 0.
"""
import io
import os
import socket
import sys
from contextlib import redirect_stdout

import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    os.environ.update({"RANK": str(rank), "LOCAL_RANK": str(rank), "WORLD_SIZE": str(world),
                       "MASTER_ADDR": "127.0.0.1", "MASTER_PORT": str(port)})
    sys.path.insert(0, ROOT)
    import bench

    w, r, local, pg = bench.dist_setup()
    assert (w, r, local) == (world, rank, rank) and pg is not None
    bench.barrier(pg)
    m = bench.max_over_ranks(pg, float(10 * (rank + 1)))
    printed = ""
    if rank != 0:
        buf = io.StringIO()
        with redirect_stdout(buf):

            class A:
                steps, warmup, ref_iters = 1, 0, 1

            bench.run_reference(A())  # returns at once: only rank 0 measures and prints
        printed = buf.getvalue()
    pg.barrier()
    pg.destroy_process_group()
    out.put((rank, m, printed))


def test_two_rank_max_and_silent_reference_rank():
    world = 2
    port = _free_port()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    by_rank = dict((r, (m, s)) for r, m, s in results)
    assert by_rank[0][0] == by_rank[1][0] == 20.0
    assert by_rank[1][1] == ""
