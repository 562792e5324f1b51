"""The multi-GPU path is replicas only (independent instances, no data-path collective):
world_size-2 gloo run of the bench's rank logic on CPU, with the oracle standing in for the
device kernels.  Each rank advances its own replica; the timing reduction takes the max."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import sys
    import time
    import datetime
    import torch
    import torch.distributed as dist
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path.insert(0, os.path.dirname(here))
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    import bench
    from dgm_in_rust_b200 import naca0012_ogrid
    from oracle.oracle import Oracle
    w, r, local = bench.dist_env()
    assert (w, r, local) == (world, rank, rank)
    o = Oracle(raw=naca0012_ogrid(16, 8), order=2, cfl=0.1, final_time=1e30, final_step=10 ** 6,
               freestream=(1.25, 0.8, 1.0, 1.0 / 1.4))
    U = o.initial_solution()
    R = o.new_state()
    dist.barrier()
    t0 = time.perf_counter()
    for _ in range(2 + rank):  # uneven work per rank
        o.rk3(R, U, o.compute_time_step(U))
    el = torch.tensor([time.perf_counter() - t0], dtype=torch.float64)
    mine = el.clone()
    dist.all_reduce(el, op=dist.ReduceOp.MAX)
    digest = torch.tensor([float(np.abs(U).sum())], dtype=torch.float64)
    allg = [torch.zeros(1, dtype=torch.float64) for _ in range(world)]
    dist.all_gather(allg, digest)
    out[rank] = (float(mine), float(el), [float(x) for x in allg])
    dist.barrier()
    dist.destroy_process_group()


def test_replicas_two_ranks_gloo():
    world, port = 2, _free_port()
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    (m0, mx0, d0), (m1, mx1, d1) = out[0], out[1]
    assert mx0 == mx1 == max(m0, m1)
    # replicas: rank 1 ran one more step than rank 0, so the replicas' states differ
    assert d0 == d1 and d0[0] != d0[1]
