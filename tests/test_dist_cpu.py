"""World-size-2 test of the bench's replica plumbing on CPU (gloo): each
rank places its own netlist (distinct seeds), the ranks meet at a barrier,
and the reported time is the max over ranks, the job count the sum."""

import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(RANK=str(rank), LOCAL_RANK=str(rank), WORLD_SIZE=str(world), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    import sys

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    import bench
    import eisenjoch_b200 as E

    d = bench.Dist(None)
    spec = bench.replica_spec(E.WORKLOADS["electro_5k_128"]["spec"], d.rank)
    nl, chip = E.synth_netlist(spec)
    d.barrier()
    t_max = d.max(1.5 + rank)      # per-rank "time"
    jobs = d.sum(3)                 # per-rank job count
    d.barrier()
    q.put((rank, spec.seed, int(nl.pin_cell[:50].sum()), t_max, jobs))
    d.close()


def test_two_rank_replicas_over_gloo():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = sorted(q.get(timeout=180) for _ in range(2))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    (r0, s0, h0, t0, j0), (r1, s1, h1, t1, j1) = out
    assert s0 != s1 and h0 != h1           # independent netlists
    assert t0 == t1 == 2.5                  # max over ranks
    assert j0 == j1 == 6                    # whole-job aggregate
