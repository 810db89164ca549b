"""The multi-GPU host logic on CPU: two gloo ranks shard the ensemble with no
data-path collective (disjoint channel sets that together form one seeded
sequence), and the timing reduction takes the slowest rank."""
import os
import socket
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    class A:
        pass
    w, r, local, pg = bench.dist_setup(A(), backend="gloo")
    plans = bench.make_plans("c3", "fp16s", w, r)
    sig = [(p.params.nx, p.params.ny, round(p.params.fluid.tau, 12)) for p in plans]
    bench.barrier(pg, local)
    mx = bench.allmax(pg, float(10 + r))
    q.put((r, sig, mx))
    pg.destroy_process_group()


def test_two_rank_sharding_and_max_timing():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict()
    for _ in range(2):
        r, sig, mx = q.get(timeout=240)
        out[r] = (sig, mx)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    sys.path.insert(0, ROOT)
    from softflow_b200 import workloads as W
    full = [(p.params.nx, p.params.ny, round(p.params.fluid.tau, 12))
            for p in W.plan_c3(n_channels=512)]
    assert out[0][0] == full[:256] and out[1][0] == full[256:]
    assert out[0][1] == out[1][1] == 11.0
