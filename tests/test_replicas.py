"""The multi-GPU path of the benchmark is replicas only: every rank
advances its own instances, the ranks meet at barriers and agree on the
slowest rank's time.  Tested with world size 2 on the gloo backend (CPU)."""
import os
import socket

import pytest
import torch.multiprocessing as tmp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    from reef3d_b200.replicas import Replicas, aggregate_rate
    r = Replicas(backend="gloo", timeout_s=30)
    r.barrier()
    slowest = r.max(1.0 + rank)          # rank 1 is slower
    rate = aggregate_rate(100.0 * (rank + 1), 2.0 * (rank + 1), r)
    r.barrier()
    r.close()
    q.put((rank, slowest, rate))


def test_two_ranks_agree_on_slowest_time_and_aggregate():
    ctx = tmp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    ps = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = sorted(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    # max over ranks of (1, 2) = 2; (100 + 200) units / max(2, 4) s = 75
    assert res == [(0, 2.0, 75.0), (1, 2.0, 75.0)]
