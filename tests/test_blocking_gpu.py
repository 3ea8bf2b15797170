"""Device blocking (vmc_blocking) against the host Blocker on the same recorded
energies: a replayed stream drives both the blocking pass and vmc_replay's per-step
record, the concatenated walker-major series and each walker's own series are blocked
on the host and compared (1e-10 relative)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DOT = ("numParticles: {N}\nnumDimensions: 2\nhamiltonian: harmonicOscillator\nomega: {omega}\n"
       "{coulomb}{slater}waveFunctionElement: gaussian\n{pade}"
       "basis: hermite\nsampling: importanceSampling\nstepLength: 0.05\nnumSteps: 1000\n")


def text(N, omega=1.0, interacting=True):
    return DOT.format(N=N, omega=omega, coulomb="interactionStyle: coulomb\n" if interacting else "",
                      slater="waveFunctionElement: slaterDeterminant\n" if N > 2 else "",
                      pade="waveFunctionElement: padeJastrow\n" if interacting else "")


def rel(a, b):
    return abs(a - b) / max(abs(b), 1e-300)


@pytest.mark.parametrize("N,W,steps,burn", [(2, 8, 700, 100), (6, 16, 1200, 80)])
def test_device_blocking_matches_host(N, W, steps, burn):
    from vmachine_b200 import Engine, block_series
    rng = np.random.default_rng(N)
    pos = rng.normal(0.0, 1.0, (W, 2 * N))
    stream = np.stack([rng.random((W, steps)), rng.normal(size=(W, steps)), rng.random((W, steps))], -1)
    with Engine(text(N), walkers=W, precision=0, compat=0) as a:
        a.init_walkers(pos)
        _, en = a.replay(stream)
    with Engine(text(N), walkers=W, precision=0, compat=0) as b:
        b.init_walkers(pos)
        b.set_replay(stream)
        r = b.blocking(steps, burn)
    n = r.samples_per_walker
    assert n == 1 << int(np.log2(steps - burn))
    parts = [en.sum(-1), en[..., 0], en[..., 1], en[..., 2]]
    for blk, series in zip((r.energy, r.kinetic, r.external, r.interaction), parts):
        s = series[:, burn:burn + n]
        h = block_series(s.reshape(-1))
        assert rel(blk.mean, h.mean) < 1e-12
        assert rel(blk.mse_mean, h.mse_mean) < 1e-10, (blk.mse_mean, h.mse_mean)
        assert blk.n_k == h.n_k
    s = parts[0][:, burn:burn + n]
    own = [block_series(s[w]) for w in range(W)]
    assert rel(r.energy_walkers.mean, np.mean([o.mean for o in own])) < 1e-12
    assert rel(r.energy_walkers.mse_mean, sum(o.mse_mean for o in own) / W ** 2) < 1e-10


def test_exact_wave_function_has_no_error():
    """Non-interacting N = 2, omega = 1 with alpha = 1: E_L = 2 at every step."""
    from vmachine_b200 import Engine
    with Engine(text(2, interacting=False), walkers=64, precision=0, compat=0) as e:
        e.set_parameters(np.array([[1.0]]))
        e.init_walkers(None, seed=3)
        r = e.blocking(2048 + 64, 64)
    assert abs(r.energy.mean - 2.0) < 1e-12
    assert r.energy.std_error < 1e-12 and r.energy_walkers.std_error < 1e-12


def test_walker_count_not_power_of_two():
    from vmachine_b200 import Engine
    with Engine(text(6), walkers=12, precision=1) as e:
        e.init_walkers(None, seed=5)
        r = e.blocking(600, 50)
    assert r.energy.n_k == 0 and r.energy.mean == -1.0
    assert r.energy_walkers.std_error > 0 and np.isfinite(r.energy_walkers.mean)
