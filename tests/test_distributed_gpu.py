"""Walker shards of real engines reproduce one engine over the whole population.

Two ranks (two processes on cuda:0, gloo for the host all-reduce) each hold half of
a 64-walker population (vmachine_b200.distributed.shard_text: walkerOffset keys the
random streams by population index) and run three iterations with
distributed.run_iteration: sample, all-reduce the totals, apply them.  One engine
over all 64 walkers runs the same three iterations.  The chains are the same walker
by walker, so the energies and the parameters after the ADAM steps agree to
rounding (only the order of the sums over walkers differs); the walkers' error bar
over ranks is the single engine's.
"""
import os
import socket
import sys

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, text, iters, out):
    sys.path.insert(0, ROOT)
    import datetime

    import torch.distributed as dist
    from vmachine_b200 import Engine
    from vmachine_b200 import distributed as vd
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    res = []
    with Engine(vd.shard_text(text, rank, world), device=0) as e:
        e.init_walkers(None, seed=5)
        for it in range(iters):
            a = vd.run_iteration(e, it)
            res.append((a.energy, a.std_error, a.walker_std_error, a.acceptance))
        out[rank] = (res, e.parameters().copy(), e.positions().copy())
    dist.barrier()
    dist.destroy_process_group()


def run_shards(text, iters, world=2):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, world, port, text, iters, out)) for r in range(world)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=300)
            assert p.exitcode == 0
        return [out[r] for r in range(world)]


@pytest.mark.parametrize("precision,tol", [("fp64", 1e-12), ("mixed", 1e-9)])
def test_shards_equal_one_engine(precision, tol):
    from vmachine_b200 import Engine
    from vmachine_b200.batch import dot_text
    # a fixed refresh cadence in mixed precision (the shards' drift tests would
    # otherwise tune on their own halves; distributed.run_iteration aligns them to the
    # most cautious one, which need not be the single engine's)
    text = dot_text(6, 0.6, 64, 300, precision, seed=7) + ("refreshInterval: 256\n" if precision == "mixed" else "")
    iters = 3
    shards = run_shards(text, iters)
    with Engine(text, device=0) as e:
        e.init_walkers(None, seed=5)
        one = []
        for it in range(iters):
            a = e.run_iteration(it)
            one.append((a.energy, a.std_error, a.walker_std_error, a.acceptance))
        theta, pos = e.parameters(), e.positions()
    (r0, t0, p0), (r1, t1, p1) = shards
    assert np.array_equal(t0, t1)  # every rank took the same step
    for (ea, sa, wa, aa), (e0, s0, w0, a0) in zip(one, r0):
        assert abs(e0 - ea) <= tol * abs(ea)
        assert abs(s0 - sa) <= 1e3 * tol * abs(sa) + 1e-15
        assert abs(w0 - wa) <= 1e3 * tol * abs(wa) + 1e-15
        assert abs(a0 - aa) <= 1e-12
    assert np.allclose(t0, theta, rtol=tol, atol=0)
    assert np.allclose(np.concatenate([p0, p1]), pos, rtol=10 * tol, atol=10 * tol)
