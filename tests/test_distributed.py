"""Multi-rank iteration glue on CPU: two gloo ranks, each with its own walker
shard, must all-reduce their sampler totals and take the identical optimiser
step that one process applying the summed totals takes (the reference's
MPI_Reduce + MPI_Bcast, src/sampler.cpp:111-187, src/system.cpp:130-135); the
walkers' error bar and status bits are those of all walkers; a rank whose pass
fails makes every rank raise (after the same collectives, so none waits).

The engines here run on the host (no GPU): fakes whose sample() returns
rank-dependent totals, and shards of one walker population whose chains the C oracle
runs on replayed random numbers; apply_sums() restates the averages and ADAM step with
the CPU checker.  Real engines on a GPU: tests/test_distributed_gpu.py.
"""
import os
import socket
import sys

import numpy as np
import torch.multiprocessing as mp

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


class FakeEngine:
    def __init__(self, rank, E=2, P=1, fail_at=None, status=0):
        from vmachine_b200.engine import Info
        self.E, self.P, self.rank = E, P, rank
        self.info = Info()
        self.info.steps_per_walker, self.info.burn_in = 100, 1
        from oracle.vmc_oracle_host import Adam
        self.theta = np.ones((E, P))
        self.opt = Adam((E, P), 0.1)
        self.fail_at, self.status, self.it = fail_at, status, 0

    def walker_energies(self):
        return 3.0 + np.random.default_rng(7 + 100 * self.rank + self.it).normal(size=5 + self.rank)

    def sample(self, iteration, steps, burn_in):
        from vmachine_b200.engine import Sums, VmcError
        self.it = iteration
        if self.fail_at == iteration:
            raise VmcError(-8, "a tensor-core completion wait gave up")
        rng = np.random.default_rng(100 * self.rank + iteration)
        s = Sums()
        s.n_samples = 1000.0
        s.n_window = 100.0
        e = 3.0 + 0.1 * rng.random()
        s.energy, s.energy2 = e * 1000, e * e * 1000 + rng.random()
        s.kinetic, s.external, s.interaction = 1000.0, 1500.0, 500.0
        s.accepts = 990.0
        s.status = self.status
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
    eng = FakeEngine(rank, status=2 if rank == 1 else 0)
    wse = []
    for it in range(3):
        a = vd.run_iteration(eng, it)
        wse.append(a["walker_std_error"])
    out[rank] = eng.theta.copy()
    out[f"wse{rank}"] = wse
    out[f"status{rank}"] = 0
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
        total, g, ge, wse, err = vd.unpack(vecs[0] + vecs[1], 2, 1)
        assert err is None
        ref.apply_sums(total, g, ge)
    assert np.allclose(theta0, ref.theta, rtol=1e-14, atol=0)


def test_pack_roundtrip():
    from vmachine_b200 import distributed as vd
    eng = FakeEngine(1)
    s, g, ge = eng.sample(0, 101, 1)
    s2, g2, ge2, _, err = vd.unpack(vd.pack(s, g, ge), 2, 1)
    assert err is None
    for f in vd.SUM_FIELDS:
        assert getattr(s2, f) == getattr(s, f)
    assert np.array_equal(g2, g) and np.array_equal(ge2, ge)


def test_walker_error_and_status_over_ranks():
    """The payload carries the walkers' mean-energy moments and status bits: the
    all-reduced vector gives the spread of all walkers' means and the OR of the bits."""
    from vmachine_b200 import distributed as vd
    a, b = FakeEngine(0, status=1), FakeEngine(1, status=8)
    va = vd.pack(*a.sample(0, 101, 1), a.walker_energies())
    vb = vd.pack(*b.sample(0, 101, 1), b.walker_energies())
    s, _, _, wse, err = vd.unpack(va + vb, 2, 1)
    m = np.concatenate([a.walker_energies(), b.walker_energies()])
    assert err is None and s.status == 9
    assert abs(wse - np.std(m, ddof=1) / np.sqrt(len(m))) < 1e-12


def test_shard_text_slices_the_population():
    from vmachine_b200 import distributed as vd
    text = "numParticles: 6\nnumWalkers: 10\nnumSteps: 1000\nwalkerOffset: 3\n"
    shards = [vd.shard_text(text, r, 3) for r in range(3)]
    got = [(int(t.split("numWalkers: ")[1].split()[0]), int(t.split("numSteps: ")[1].split()[0]),
            int(t.split("walkerOffset: ")[1].split()[0])) for t in shards]
    assert got == [(4, 400, 0), (3, 300, 4), (3, 300, 7)]
    assert all(t.count("walkerOffset") == 1 and t.startswith("numParticles: 6") for t in shards)


def _failing_rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from vmachine_b200 import distributed as vd
    from vmachine_b200.engine import VmcError
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    eng = FakeEngine(rank, fail_at=1 if rank == 1 else None)
    codes = []
    for it in range(3):
        try:
            vd.run_iteration(eng, it)
            codes.append(0)
        except VmcError as exc:
            codes.append(exc.code)
    out[rank] = codes
    dist.barrier()
    dist.destroy_process_group()


def test_a_failing_rank_fails_every_rank():
    """Rank 1's pass fails at iteration 1: both ranks still take the iteration's
    collectives, both raise, and both go on to iteration 2 together."""
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_failing_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        assert out[0] == [0, -8, 0] and out[1] == [0, -8, 0]


class OracleShard:
    """A slice of one walker population run by the C oracle (oracle/vmc_oracle.c),
    with the engine's interface as distributed.run_iteration uses it.  Every walker
    has its own replayed random stream, the population's row for that walker, so a
    slice walks exactly the chains the whole population walks."""

    STEPS, BURN = 200, 2

    def __init__(self, lo, hi, n_walkers=6, iterations=3):
        sys.path.insert(0, HERE)
        sys.path.insert(0, ROOT)
        from oracle.vmc_oracle_host import Adam
        from oracle_bind import GAUSSIAN, PADE, Oracle, SystemSpec
        from vmachine_b200.engine import Info
        self.spec = SystemSpec(N=2, elements=(GAUSSIAN, PADE), step=0.05, omega=1.0)
        self.O = Oracle()
        rng = np.random.default_rng(11)
        D, per = self.spec.D, self.STEPS + self.BURN
        pos = rng.normal(0.0, 1.0, (n_walkers, D))
        stream = np.empty((n_walkers, per * iterations, 3))
        stream[..., 0] = rng.random(stream.shape[:2])
        stream[..., 1] = rng.normal(size=stream.shape[:2])
        stream[..., 2] = rng.random(stream.shape[:2])
        self.pos, self.stream = pos[lo:hi].copy(), stream[lo:hi]
        self.theta = np.array([[1.0], [0.5]])
        self.E, self.P = self.theta.shape
        self.f = np.stack([self.O.quantum_force(self.spec, self.theta, p) for p in self.pos])
        self.opt = Adam(self.theta.shape, 0.05)
        self.info = Info()
        self.info.steps_per_walker, self.info.burn_in, self.info.precision = self.STEPS, self.BURN, 0
        self.off, self.means = 0, None

    def sample(self, iteration, steps, burn_in):
        from vmachine_b200.engine import Sums
        W = len(self.pos)
        out = self.O.run(self.spec, self.theta, self.pos, self.f, steps, burn_in, iteration,
                         self.opt.batches, stream=self.stream[:, self.off:self.off + steps], want_steps=False)
        self.off += steps
        per_walker = out["sums"]
        n = steps - burn_in
        self.means = per_walker[:, 0] / n
        S = per_walker.sum(0)
        s = Sums()
        for i, f in enumerate(("energy", "energy2", "kinetic", "kinetic2", "external", "external2",
                               "interaction", "interaction2", "accepts")):
            setattr(s, f, S[i])
        s.n_samples, s.n_window = W * n, W * (n // self.opt.batches)
        ep = self.E * self.P
        return s, S[9:9 + ep].reshape(self.E, self.P), S[9 + ep:9 + 2 * ep].reshape(self.E, self.P)

    def walker_energies(self):
        return self.means

    def apply_sums(self, s, g, ge):
        from oracle.vmc_oracle_host import averages, energy_gradient
        vec = [s.energy, s.energy2, s.kinetic, s.kinetic2, s.external, s.external2, s.interaction,
               s.interaction2, s.accepts]
        avg = averages(np.concatenate([vec, g.ravel(), ge.ravel()]), s.n_samples, s.n_window,
                       (self.E, self.P))
        self.theta = self.theta - self.opt.update(energy_gradient(avg))
        return avg


def _oracle_rank(rank, world, port, out):
    sys.path.insert(0, ROOT)
    import torch.distributed as dist
    from vmachine_b200 import distributed as vd
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    eng = OracleShard(3 * rank, 3 * rank + 3)
    hist = []
    for it in range(3):
        a = vd.run_iteration(eng, it)
        hist.append((a["energy"], a["walker_std_error"]))
    out[rank] = (eng.theta.copy(), hist)
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_ranks_of_oracle_chains_equal_one_population():
    """Two ranks, each running three walkers' chains in the C oracle, all-reduce their
    totals through distributed.run_iteration: every iteration's energy and walker
    error bar and the parameters after three ADAM steps equal those of one process
    running all six walkers (the reference's one-rank computeTotals and update)."""
    sys.path.insert(0, ROOT)
    from vmachine_b200 import distributed as vd
    ctx = mp.get_context("spawn")
    with ctx.Manager() as mgr:
        out = mgr.dict()
        port = _free_port()
        procs = [ctx.Process(target=_oracle_rank, args=(r, 2, port, out)) for r in range(2)]
        for p in procs:
            p.start()
        for p in procs:
            p.join(timeout=120)
            assert p.exitcode == 0
        (theta0, hist0), (theta1, hist1) = out[0], out[1]
    assert np.array_equal(theta0, theta1) and hist0 == hist1
    one = OracleShard(0, 6)
    for it in range(3):
        a = vd.run_iteration(one, it)
        assert abs(a["energy"] - hist0[it][0]) <= 1e-13 * abs(a["energy"])
        # the spread from summed moments cancels: a few units in the 12th digit
        assert abs(a["walker_std_error"] - hist0[it][1]) <= 1e-10 * a["walker_std_error"]
    assert np.allclose(theta0, one.theta, rtol=1e-12, atol=0)
