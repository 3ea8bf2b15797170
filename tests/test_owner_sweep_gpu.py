"""The owner form of the production dot sweep (vmc_owner_sweep.cuh).

One walker per warp, each lane holding two particles' positions, derivative vectors
and Pade gradients in registers.  It is the default production sweep of the dots
that keep one walker per warp (N = 42 and 56) and runs N = 20 and 30 on request
(`sweepForm: owner`).  The FP64 form is held to the C oracle on the walkers' own
Philox streams (final positions, accept counts and sampled energies, as the staged
form is in test_gpu_parity.py); the mixed form is held to the staged mixed sweep on
the same streams, and whole FP64 iterations (ADAM steps included) to the staged FP64
sweep.
"""
import numpy as np
import pytest

from oracle_bind import GAUSSIAN, PADE, SLATER, Oracle, SystemSpec

pytestmark = pytest.mark.gpu

OMEGA = {20: 0.5, 30: 0.5, 42: 0.3, 56: 0.28}


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def spec_for(n, walkers, steps, compat, form, step=0.01):
    return SystemSpec(N=n, omega=OMEGA[n], elements=(SLATER, GAUSSIAN, PADE), step=step,
                      num_steps=walkers * steps, quirks=SystemSpec().quirks if compat else 0,
                      extra=[f"sweepForm: {form}"])


@pytest.mark.parametrize("n,walkers", [(20, 19), (30, 9), (42, 7), (56, 5)])
@pytest.mark.parametrize("compat", [1, 0])
def test_owner_sweep_matches_oracle(n, walkers, compat):
    """FP64 owner sweep on Philox streams against the oracle: 1e-11 final positions,
    identical accept counts, 1e-10 sampled energy sums."""
    from vmachine_b200 import Engine
    from vmachine_b200.engine import SWEEP_OWNER
    steps, seed = 300, 4321
    spec = spec_for(n, walkers, steps, compat, "owner")
    rng = np.random.default_rng(n)
    pos = rng.normal(0, 1 / np.sqrt(OMEGA[n]), size=(walkers, spec.D))
    theta = np.array([[0.0], [1.0], [0.5]])
    with Engine(spec.input_in(), walkers=walkers, precision=0, compat=compat) as eng:
        assert eng.info.sweep_form == SWEEP_OWNER
        eng.set_parameters(theta)
        eng.init_walkers(pos, seed=seed)
        s, _, _ = eng.sample(0, steps, 0)
        final = eng.positions()
    O = Oracle()
    p = pos.copy()
    f = np.stack([O.quantum_force(spec, theta, pos[w]) for w in range(walkers)])
    out = O.run(spec, theta, p, f, steps, 0, 0, 10, stream=None, seed=seed, counter=np.zeros(walkers, np.uint64))
    assert rel(final, p) < 1e-11
    assert abs(s.accepts - out["sums"][:, 8].sum()) < 0.5
    assert abs(s.energy - out["sums"][:, 0].sum()) < 1e-10 * abs(out["sums"][:, 0].sum())


@pytest.mark.parametrize("n,walkers", [(20, 19), (56, 5)])
def test_owner_sweep_drift_limit_matches_oracle(n, walkers):
    """The corrected mode's drift limiter (driftLimit: 0.5) in the FP64 owner sweep
    against the oracle on Philox streams, as above."""
    from vmachine_b200 import Engine
    from vmachine_b200.engine import SWEEP_OWNER
    steps, seed = 300, 1234
    spec = spec_for(n, walkers, steps, 0, "owner")
    spec.drift_limit = 0.5
    rng = np.random.default_rng(n + 1)
    pos = rng.normal(0, 1 / np.sqrt(OMEGA[n]), size=(walkers, spec.D))
    theta = np.array([[0.0], [1.0], [0.5]])
    with Engine(spec.input_in(), walkers=walkers, precision=0, compat=0) as eng:
        assert eng.info.sweep_form == SWEEP_OWNER
        eng.set_parameters(theta)
        eng.init_walkers(pos, seed=seed)
        s, _, _ = eng.sample(0, steps, 0)
        final = eng.positions()
    O = Oracle()
    p = pos.copy()
    f = np.stack([O.quantum_force(spec, theta, pos[w]) for w in range(walkers)])
    out = O.run(spec, theta, p, f, steps, 0, 0, 10, stream=None, seed=seed, counter=np.zeros(walkers, np.uint64))
    assert rel(final, p) < 1e-11
    assert abs(s.accepts - out["sums"][:, 8].sum()) < 0.5
    assert abs(s.energy - out["sums"][:, 0].sum()) < 1e-10 * abs(out["sums"][:, 0].sum())


@pytest.mark.parametrize("n", [20, 56])
@pytest.mark.parametrize("compat", [1, 0])
def test_owner_mixed_tracks_staged(n, compat):
    """Mixed precision, same Philox streams: the owner form's sampled energy, accept
    count and gradient sums against the staged form's.  The two run their FP32
    arithmetic in different orders (and the owner form sums its FP32 samples shifted,
    folded into FP64 every 32 steps), so a near-tie accept decision can flip, after
    which that walker's chain decorrelates: most walkers end at the same positions,
    and the sums over all walkers agree to 1e-5."""
    from vmachine_b200 import Engine
    W, steps = 64, 1000
    res = {}
    for form in ("staged", "owner"):
        spec = spec_for(n, W, steps, compat, form, step=0.005)
        with Engine(spec.input_in() + "seed: 7\n", walkers=W, precision=1, compat=compat) as eng:
            eng.init_walkers(None, seed=7)
            s, g, ge = eng.sample(0, steps, 10)
            res[form] = (s, np.array(g), np.array(ge), eng.positions())
    (sa, ga, gea, pa), (sb, gb, geb, pb) = res["staged"], res["owner"]
    assert abs(sb.energy - sa.energy) < 1e-5 * abs(sa.energy)
    assert abs(sb.energy2 - sa.energy2) < 1e-5 * abs(sa.energy2)
    assert abs(sb.accepts - sa.accepts) <= 1e-3 * sa.n_samples
    assert rel(gb, ga) < 1e-4 and rel(geb, gea) < 1e-4
    same = [rel(pb[w], pa[w]) < 1e-4 for w in range(W)]
    assert np.mean(same) >= 0.9, np.mean(same)


@pytest.mark.parametrize("compat", ["reference", "corrected"])
def test_owner_iterations_match_staged_fp64(compat):
    """Three FP64 iterations with ADAM steps (N = 56, 37 walkers): energies and
    parameters of the owner form equal the staged form's."""
    from vmachine_b200 import Engine
    from vmachine_b200.batch import dot_text
    text = dot_text(56, 0.28, 37, 300, "fp64", seed=11, compat=compat)
    out = {}
    for form in ("staged", "owner"):
        with Engine(text + f"sweepForm: {form}\n") as e:
            e.init_walkers(None, seed=3)
            out[form] = [(e.run_iteration(it).energy, e.parameters().copy()) for it in range(3)]
    for (ea, ta), (eb, tb) in zip(out["staged"], out["owner"]):
        assert abs(eb - ea) < 1e-11 * abs(ea)
        assert np.allclose(tb, ta, rtol=1e-9, atol=0)


def test_sweep_form_selection():
    """Owner form by default where one walker per warp remains (N = 42, 56), staged on
    request; N = 20 and 30 keep two walkers per warp unless the owner form is asked
    for; smaller dots have no owner form."""
    from vmachine_b200 import Engine, VmcError
    from vmachine_b200.batch import dot_text
    from vmachine_b200.engine import SWEEP_OWNER, SWEEP_STAGED
    for N, expect in ((12, SWEEP_STAGED), (20, SWEEP_STAGED), (30, SWEEP_STAGED), (42, SWEEP_OWNER),
                      (56, SWEEP_OWNER)):
        for prec in ("mixed", "fp64"):
            with Engine(dot_text(N, 0.5, 64, 10, prec), device=0) as e:
                assert e.info.sweep_form == expect, (N, prec)
    with Engine(dot_text(56, 0.5, 64, 10) + "sweepForm: staged\n", device=0) as e:
        assert e.info.sweep_form == SWEEP_STAGED and e.info.walkers_per_warp == 1
    with Engine(dot_text(20, 0.5, 64, 10) + "sweepForm: owner\n", device=0) as e:
        assert e.info.sweep_form == SWEEP_OWNER and e.info.walkers_per_warp == 1
    with pytest.raises(VmcError):
        Engine(dot_text(12, 0.5, 64, 10) + "sweepForm: owner\n", device=0)
