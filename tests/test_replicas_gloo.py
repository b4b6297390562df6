"""Multi-GPU is replicas only: every rank analyses and factors its own copy
of the system, with no collective on the data path; the only collectives are
the barrier and the max over ranks of the timed region.  Exercised here with
world_size 2 on the gloo backend (CPU processes): each rank builds the
benchmark system and its symbolic factor independently, the structures agree
across ranks, and bench.py's max-over-ranks returns the slowest rank's time
on every rank."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out):
    import datetime
    import sys
    import torch.distributed as dist
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, root)
    import bench
    import taucs_b200 as tb
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    A, perm, iperm, P, B = bench.make_system("mixed80", 12)
    F = tb.factor_symbolic(P)
    inf = F.info()
    slowest = bench.max_over_ranks_of(dist, 10.0 + rank, "cpu")
    dist.barrier()
    dist.destroy_process_group()
    out.put((rank, inf.flops, inf.n_live, int(np.sum(perm)), slowest))


@pytest.mark.timeout(300)
def test_two_replicas_gloo():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=240) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, f0, l0, p0, s0), (r1, f1, l1, p1, s1) = res
    assert (f0, l0, p0) == (f1, l1, p1)       # identical, independently built replicas
    assert s0 == s1 == 11.0                    # max over ranks seen by every rank
