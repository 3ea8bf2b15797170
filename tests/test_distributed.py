"""Multi-rank iteration glue on CPU: two gloo ranks, each with its own walker
shard, must all-reduce their sampler totals and take the identical optimiser
step that one process applying the summed totals takes (the reference's
MPI_Reduce + MPI_Bcast, src/sampler.cpp:111-187, src/system.cpp:130-135).

The engines here are host fakes (no GPU): sample() returns rank-dependent
totals; apply_sums() restates the averages and ADAM step with the CPU checker.
"""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


class FakeEngine:
    def __init__(self, rank, E=2, P=1):
        from vmachine_b200.engine import Info
        self.E, self.P, self.rank = E, P, rank
        self.info = Info()
        self.info.steps_per_walker, self.info.burn_in = 100, 1
        from oracle.vmc_oracle_host import Adam
        self.theta = np.ones((E, P))
        self.opt = Adam((E, P), 0.1)

    def sample(self, iteration, steps, burn_in):
        from vmachine_b200.engine import Sums
        rng = np.random.default_rng(100 * self.rank + iteration)
        s = Sums()
        s.n_samples = 1000.0
        s.n_window = 100.0
        e = 3.0 + 0.1 * rng.random()
        s.energy, s.energy2 = e * 1000, e * e * 1000 + rng.random()
        s.kinetic, s.external, s.interaction = 1000.0, 1500.0, 500.0
        s.accepts = 990.0
        g = rng.normal(size=(self.E, self.P)) * 100
        ge = g * e + rng.normal(size=(self.E, self.P))
        return s, g, ge

    def apply_sums(self, s, g, ge):
        from oracle.vmc_oracle_host import averages, energy_gradient
        vec = [s.energy, s.energy2, s.kinetic, 0, s.external, 0, s.interaction, 0, s.accepts]
        vec = np.concatenate([vec, g.ravel(), ge.ravel()])
        avg = averages(vec, s.n_samples, s.n_window, (self.E, self.P))
        self.theta = self.theta - self.opt.update(energy_gradient(avg))
        return avg


def _rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from vmachine_b200 import distributed as vd
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    eng = FakeEngine(rank)
    for it in range(3):
        vd.run_iteration(eng, it)
    out[rank] = eng.theta.copy()
    dist.barrier()
    dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_two_gloo_ranks_take_the_same_step():
    sys.path.insert(0, ROOT)
    from vmachine_b200 import distributed as vd
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        theta0, theta1 = out[0], out[1]
    assert np.array_equal(theta0, theta1)
    # single process applying the summed totals of both shards
    ref = FakeEngine(0)
    shards = [FakeEngine(0), FakeEngine(1)]
    for it in range(3):
        vecs = [vd.pack(*sh.sample(it, 101, 1)) for sh in shards]
        total, g, ge = vd.unpack(vecs[0] + vecs[1], 2, 1)
        ref.apply_sums(total, g, ge)
    assert np.allclose(theta0, ref.theta, rtol=1e-14, atol=0)


def test_pack_roundtrip():
    from vmachine_b200 import distributed as vd
    eng = FakeEngine(1)
    s, g, ge = eng.sample(0, 101, 1)
    s2, g2, ge2 = vd.unpack(vd.pack(s, g, ge), 2, 1)
    for f in vd.SUM_FIELDS:
        assert getattr(s2, f) == getattr(s, f)
    assert np.array_equal(g2, g) and np.array_equal(ge2, ge)
