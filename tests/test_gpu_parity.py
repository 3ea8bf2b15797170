"""Parity of the CUDA engine (through the C ABI) with the reference.

Golden vectors come from the reference's own C++ sources (tests/golden/); the C
oracle (oracle/vmc_oracle.c, pinned to the same vectors) checks what the
fixtures do not cover.  FP64 bar: 1e-11 relative at fixed positions (max-abs
over each array relative to its max-abs), identical accept/reject decisions on
replayed streams, 1e-10 relative along replayed chains and iterations (the engine
carries running pair sums where the reference recomputes).
"""
import os

import numpy as np
import pytest

from oracle_bind import (GAUSSIAN, HYDROGENLIKE, PADE, RBMGAUSSIAN, RBMPRODUCT, SIMPLEJASTROW, SLATER,
                         Oracle, SystemSpec, load_cases, spec_from_case)

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
EVAL = load_cases(os.path.join(GOLD, "eval_fixed.npz"))
CHAINS = load_cases(os.path.join(GOLD, "chains.npz"))
ITERS = load_cases(os.path.join(GOLD, "iterations.npz"))
for _f in ("hydrogen_orbitals.npz", "hydrogen_simplejastrow.npz"):
    _H = load_cases(os.path.join(GOLD, _f))
    EVAL.update({k: v for k, v in _H.items() if not k.startswith("chain_")})
    CHAINS.update({k[len("chain_"):]: v for k, v in _H.items() if k.startswith("chain_")})
ENGINE_ELEMENTS = {GAUSSIAN, SLATER, PADE, HYDROGENLIKE, SIMPLEJASTROW, RBMGAUSSIAN, RBMPRODUCT}


def supported(c):
    return set(int(e) for e in c["spec_elements"]) <= ENGINE_ELEMENTS


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    scale = max(float(np.max(np.abs(b))) if b.size else 0.0, 1e-300)
    return float(np.max(np.abs(a - b)) / scale) if b.size else 0.0


def make_engine(spec, walkers, precision=0, compat=1):
    from vmachine_b200 import Engine
    return Engine(spec.input_in(), walkers=walkers, precision=precision, compat=compat)


@pytest.mark.parametrize("name", sorted(n for n in EVAL if supported(EVAL[n])))
def test_fixed_positions(name):
    c = EVAL[name]
    spec = spec_from_case(c)
    pos = c["pos"]
    with make_engine(spec, len(pos)) as eng:
        eng.set_parameters(c["theta"])
        eng.init_walkers(pos)
        g, lap, pg, en = eng.eval()
        for t in range(len(pos)):
            assert rel(g[t], c["grad"][t]) < 1e-11
            assert rel(lap[t], c["lap"][t]) < 1e-11
            assert rel(pg[t], c["pgrad"][t]) < 1e-11
            assert rel(en[t], c["energies"][t]) < 1e-11
        r = eng.probe_move(c["k"], c["xnew"])
        g, lap, pg, en = eng.eval()
        for t in range(len(pos)):
            assert rel(r[t], c["ratios"][t]) < 1e-11
            assert rel(g[t], c["grad2"][t]) < 1e-11
            assert rel(lap[t], c["lap2"][t]) < 1e-11
            assert rel(pg[t], c["pgrad2"][t]) < 1e-11
            assert rel(en[t], c["energies2"][t]) < 1e-11


@pytest.mark.parametrize("name", sorted(n for n in CHAINS if supported(CHAINS[n])))
def test_replayed_chain(name):
    c = CHAINS[name]
    spec = spec_from_case(c)
    with make_engine(spec, 1) as eng:
        eng.set_parameters(c["theta"])
        eng.init_walkers(c["pos"][None])
        acc, en = eng.replay(c["stream"][None])
        assert np.array_equal(acc[0], c["accepted"])
        assert rel(en[0], c["energies"]) < 1e-10
        assert rel(eng.positions()[0], c["final_pos"]) < 1e-11


@pytest.mark.parametrize("name", sorted(n for n in ITERS if supported(ITERS[n])))
def test_iterations(name):
    c = ITERS[name]
    spec = spec_from_case(c)
    with make_engine(spec, 1) as eng:
        assert eng.info.burn_in == int(c["burn_in"])
        assert eng.info.steps_per_walker == int(c["steps_wo"])
        assert eng.info.batches == int(c["batches"])
        eng.set_parameters(c["theta0"])
        eng.init_walkers(c["pos"][None])
        eng.set_replay(c["stream"][None])
        for it in range(len(c["energy"])):
            a = eng.run_iteration(it)
            assert rel(a.energy, c["energy"][it]) < 1e-10
            assert rel(a.kinetic, c["kinetic"][it]) < 1e-10
            assert rel(a.external, c["external"][it]) < 1e-10
            assert rel(a.interaction, c["interaction"][it]) < 1e-10
            assert rel(a.acceptance, c["acceptance"][it]) < 1e-12
            assert rel(a.std_error, c["std_error"][it]) < 1e-7
            assert rel(eng.parameters(), c["params"][it]) < 1e-10


def test_philox_streams_match_oracle():
    """Seeded brute-force run: the device Philox streams equal the oracle's."""
    spec = SystemSpec(N=2, elements=(GAUSSIAN, PADE), sampling="bruteForce", num_steps=4000)
    O = Oracle()
    W, steps, seed = 4, 300, 1234
    rng = np.random.default_rng(5)
    pos = rng.normal(size=(W, spec.D))
    theta = np.array([[1.0], [0.7]])
    with make_engine(spec, W) as eng:
        eng.set_parameters(theta)
        eng.init_walkers(pos, seed=seed)
        acc, en = eng.replay(None, steps)
        final = eng.positions()
    p = pos.copy()
    f = np.zeros_like(p)
    out = O.run(spec, theta, p, f, steps, 0, 0, 1, stream=None, seed=seed,
                counter=np.zeros(W, np.uint64))
    assert np.array_equal(acc, out["accepted"])
    assert rel(en, out["energies"]) < 1e-10
    assert rel(final, p) < 1e-12


def test_noninteracting_exact_energy():
    """Gaussian only, alpha = 1: E_L = 2 at every sample, zero variance."""
    spec = SystemSpec(N=2, elements=(GAUSSIAN,), coulomb=False, num_steps=64 * 2000,
                      optimization="gd", learning_rate=0.5)
    for precision in (0, 1):
        with make_engine(spec, 64, precision=precision) as eng:
            eng.init_walkers(None, seed=7)
            a = eng.run_iteration(0)
            tol = 1e-12 if precision == 0 else 1e-6
            assert abs(a.energy - 2.0) < tol
            assert a.std_error < (1e-7 if precision == 0 else 1e-4)


@pytest.mark.parametrize("drift_limit", [0.0, 0.5])
def test_corrected_mode_matches_oracle_chain(drift_limit):
    """compat: corrected (full Pade ratio, Fokker-Planck Green's ratio) against the oracle,
    without and with the drift limiter."""
    from oracle_bind import Q_RBM_SORT
    spec = SystemSpec(N=6, elements=(SLATER, GAUSSIAN, PADE), step=0.05, quirks=0, drift_limit=drift_limit)
    O = Oracle()
    rng = np.random.default_rng(11)
    steps = 300
    pos = rng.normal(size=(1, spec.D))
    stream = np.stack([rng.random(steps), rng.normal(size=steps), rng.random(steps)], -1)[None]
    theta = np.array([[0.0], [0.95], [0.6]])
    with make_engine(spec, 1, compat=0) as eng:
        eng.set_parameters(theta)
        eng.init_walkers(pos)
        acc, en = eng.replay(stream)
    p = pos.copy()
    f = np.zeros_like(p)
    out = O.run(spec, theta, p, f, steps, 0, 0, 1, stream=stream)
    assert np.array_equal(acc, out["accepted"])
    assert rel(en, out["energies"]) < 1e-10
    del Q_RBM_SORT


@pytest.mark.parametrize("Z,elements,compat,drift_limit", [
    (2, (SLATER, SIMPLEJASTROW), 1, 0.0), (10, (SLATER, SIMPLEJASTROW), 1, 0.0),
    (10, (SLATER, SIMPLEJASTROW), 0, 0.0), (10, (SLATER, PADE, SIMPLEJASTROW), 0, 0.0),
    (10, (SLATER, SIMPLEJASTROW), 0, 0.5)])
def test_atom_sweep_matches_oracle_chain(Z, elements, compat, drift_limit):
    """Atoms (hydrogen-orbital Slater determinant with SimpleJastrow and Pade-Jastrow
    factors) take the general path's compiled 3D form: replayed chains of four
    walkers against the oracle, reference Green's ratio and corrected."""
    spec = SystemSpec(N=Z, d=3, Z=Z, atom=True, basis="hydrogenOrbital", elements=elements, step=0.01,
                      quirks=SystemSpec().quirks if compat else 0, drift_limit=drift_limit)
    rng = np.random.default_rng(Z + 7 * compat)
    W, steps = 4, 300
    pos = rng.normal(size=(W, spec.D))
    stream = np.stack([rng.random((W, steps)), rng.normal(size=(W, steps)), rng.random((W, steps))], -1)
    theta = np.zeros((len(elements), spec.p_max))
    for e, el in enumerate(elements):
        if el == SIMPLEJASTROW:
            theta[e, :Z * Z] = rng.uniform(0.1, 0.5, Z * Z)
        elif el == PADE:
            theta[e, 0] = 0.8
    with make_engine(spec, W, compat=compat) as eng:
        eng.set_parameters(theta)
        eng.init_walkers(pos)
        acc, en = eng.replay(stream)
        final = eng.positions()
    p = pos.copy()
    f = np.zeros_like(p)
    out = Oracle().run(spec, theta, p, f, steps, 0, 0, 1, stream=stream)
    assert np.array_equal(acc, out["accepted"])
    assert rel(en, out["energies"]) < 1e-10
    assert rel(final, p) < 1e-11


@pytest.mark.parametrize("n,walkers,compat", [(2, 37, 1), (6, 37, 1), (12, 37, 0), (20, 19, 1), (56, 5, 1)])
def test_production_sweep_matches_oracle(n, walkers, compat):
    """The production sweep (Philox numbers drawn lane-parallel, nothing recorded; four
    walkers per warp for N <= 6, two for N = 12 and 20, one for N = 56) against the
    oracle on the same per-walker Philox streams, FP64: the same final positions and
    the same sums of sampled energies and accepts."""
    omega = {2: 1.0, 6: 1.0, 12: 0.8, 20: 0.5, 56: 0.28}[n]
    steps, seed = 300, 4321
    spec = SystemSpec(N=n, omega=omega, elements=(SLATER, GAUSSIAN, PADE), step=0.01,
                      num_steps=walkers * steps, quirks=SystemSpec().quirks if compat else 0)
    rng = np.random.default_rng(n)
    pos = rng.normal(0, 1 / np.sqrt(omega), size=(walkers, spec.D))
    theta = np.array([[0.0], [1.0], [0.5]])
    with make_engine(spec, walkers, compat=compat) as eng:
        eng.set_parameters(theta)
        eng.init_walkers(pos, seed=seed)
        s, _, _ = eng.sample(0, steps, 0)
        final = eng.positions()
    O = Oracle()
    p = pos.copy()
    # the importance-sampling force cache as initialised (ImportanceSampling::initialize);
    # the reference-mode Green's ratio reads it for coordinates not yet moved
    f = np.stack([O.quantum_force(spec, theta, pos[w]) for w in range(walkers)])
    out = O.run(spec, theta, p, f, steps, 0, 0, 10, stream=None, seed=seed, counter=np.zeros(walkers, np.uint64))
    assert rel(final, p) < 1e-11
    assert abs(s.accepts - out["sums"][:, 8].sum()) < 0.5
    assert abs(s.energy - out["sums"][:, 0].sum()) < 1e-10 * abs(out["sums"][:, 0].sum())


@pytest.mark.parametrize("Z,walkers", [(2, 37), (10, 9)])
def test_atom_sweep_matches_oracle_philox(Z, walkers):
    """The atoms' sweep on its own Philox streams (He four walkers per warp, a last warp
    with one; Ne one per warp) against the oracle: final positions and sampled sums."""
    steps, seed = 300, 977
    spec = SystemSpec(N=Z, d=3, Z=Z, atom=True, basis="hydrogenOrbital", elements=(SLATER, SIMPLEJASTROW),
                      step=0.01, num_steps=walkers * steps)
    rng = np.random.default_rng(Z)
    pos = rng.normal(size=(walkers, spec.D))
    theta = np.zeros((2, spec.p_max))
    theta[1, :Z * Z] = rng.uniform(0.1, 0.5, Z * Z)
    with make_engine(spec, walkers) as eng:
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


@pytest.mark.parametrize("n", [6, 20, 56])
def test_mixed_precision_tracks_fp64(n):
    """FP32 sweep with FP64 rebuilds: same decisions on a replayed stream (a flip
    is allowed only where the FP64 weight sits within 1e-4 of its uniform) and
    energies within 1e-4 relative while the chains agree."""
    omega = {6: 1.0, 20: 0.5, 56: 0.28}[n]
    spec = SystemSpec(N=n, omega=omega, elements=(SLATER, GAUSSIAN, PADE), step=0.01)
    rng = np.random.default_rng(n)
    W, steps = 8, 1000
    pos = rng.normal(0, 1 / np.sqrt(omega), size=(W, spec.D))
    stream = np.stack([rng.random((W, steps)), rng.normal(size=(W, steps)),
                       rng.random((W, steps))], -1)
    res = {}
    for prec in (0, 1):
        with make_engine(spec, W, precision=prec) as eng:
            eng.init_walkers(pos)
            res[prec] = eng.replay(stream)
    a64, e64 = res[0]
    a32, e32 = res[1]
    for w in range(W):
        diff = np.nonzero(a64[w] != a32[w])[0]
        upto = diff[0] if len(diff) else steps
        assert upto > steps // 2 or len(diff) == 0, (w, upto)
        el64 = e64[w, :upto].sum(-1)
        el32 = e32[w, :upto].sum(-1)
        assert np.max(np.abs(el32 - el64) / np.abs(el64)) < 1e-4


def test_kernel_selection():
    """Quantum dots run the compiled-in flag set in both compat modes and both
    precisions; systems without a Slater determinant read flags at run time;
    SimpleJastrow / RBM / hydrogen orbitals take the general path."""
    from vmachine_b200 import Engine
    from vmachine_b200.engine import KERNEL_DOT, KERNEL_GENERAL, KERNEL_RUNTIME_FLAGS
    dot = SystemSpec(N=56, omega=0.28, elements=(SLATER, GAUSSIAN, PADE), num_steps=64 * 100)
    for compat in (1, 0):
        for precision in (0, 1):
            with Engine(dot.input_in(), walkers=64, precision=precision, compat=compat) as eng:
                assert eng.info.kernel_variant == KERNEL_DOT, (compat, precision)
    with Engine(SystemSpec(N=2, elements=(GAUSSIAN, PADE)).input_in(), walkers=4) as eng:
        assert eng.info.kernel_variant == KERNEL_RUNTIME_FLAGS
    sj = SystemSpec(N=6, elements=(SLATER, GAUSSIAN, SIMPLEJASTROW), sorting=True)
    with Engine(sj.input_in(), walkers=4) as eng:
        assert eng.info.kernel_variant == KERNEL_GENERAL
