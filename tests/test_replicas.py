"""Replica parallelism on CPU with the gloo backend, world size 2: each rank runs its own
replica (own seed, own fields, oracle Dslash as the per-rank work), no data crosses ranks, and
the job rate is the sum of the work over the max of the times, identical on every rank."""
import os
import socket

import numpy as np
import pytest


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank_main(rank, world, port, q):
    import sys
    import time
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    sys.path.insert(0, os.path.join(root, "rhmc-on-gpu_b200"))
    sys.path.insert(0, os.path.join(root, "oracle"))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    import datetime
    import torch.distributed as dist
    from rhmc_b200 import fields as F
    from rhmc_b200 import replicas as RP
    import oracle
    dist.init_process_group("gloo", timeout=datetime.timedelta(seconds=60))
    r, w, _ = RP.world()
    dims = (4, 4, 4, 4)
    u = F.random_links(dims, seed=RP.replica_seed(1001, r))
    x = F.random_spinor(dims, seed=RP.replica_seed(2002, r))
    orc = oracle.Oracle(dims)
    t0 = time.perf_counter()
    y = orc.deo(u, orc.doe(u, x))
    dt = time.perf_counter() - t0 + 0.01 * (r + 1)  # ranks take different times
    rate = RP.job_rate(1.0, dt, dist)
    tmax = RP.max_over_ranks(dt, dist)
    dist.barrier()
    dist.destroy_process_group()
    q.put((r, w, float(np.abs(y).sum()), dt, rate, tmax))


@pytest.mark.timeout(120)
def test_gloo_two_replicas():
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=100) for _ in procs)
    for p in procs:
        p.join(timeout=30)
        assert p.exitcode == 0
    (r0, w0, s0, t0, rate0, m0), (r1, w1, s1, t1, rate1, m1) = res
    assert (r0, r1, w0, w1) == (0, 1, 2, 2)
    assert s0 != s1  # independent replicas: different seeds, different fields
    assert m0 == m1 == max(t0, t1)
    assert rate0 == rate1 and abs(rate0 - 2.0 / max(t0, t1)) < 1e-9 * rate0


def test_single_process_fallback():
    from rhmc_b200 import replicas as RP
    assert RP.max_over_ranks(3.0) == 3.0
    assert RP.job_rate(10.0, 2.0) == 5.0
    assert RP.replica_seed(5, 0) == 5 and RP.replica_seed(5, 1) != 5
