"""The learned MLP Jastrow on the GPU (through the C ABI) against the FP64 oracle
(oracle/mlp_jastrow.py, itself checked by finite differences).

The engine evaluates the networks in FP32 with bfloat16 weights, so the bar is
relative (max-abs over an array, relative to its max-abs): 2e-5 for J-derived
gradients, Laplacians, energies and ratios, 1e-4 for dJ/dtheta (sums over pairs
of FP32 products).  The Slater and Gaussian parts come from the C oracle at 1e-11.
"""
import numpy as np
import pytest

from oracle import mlp_jastrow as mj
from oracle_bind import GAUSSIAN, SLATER, Oracle, SystemSpec

pytestmark = pytest.mark.gpu


def config(N, omega=1.0, sampling="importanceSampling", steps=1000, extra=()):
    lines = [f"numParticles: {N}", "numDimensions: 2", "hamiltonian: harmonicOscillator",
             f"omega: {omega!r}", "interactionStyle: coulomb",
             "waveFunctionElement: slaterDeterminant", "waveFunctionElement: gaussian",
             "waveFunctionElement: mlpJastrow", "basis: hermite", f"sampling: {sampling}",
             "stepLength: 0.05", "optimization: adam", "learningRate: 0.01", f"numSteps: {steps}"]
    return "\n".join(list(lines) + list(extra)) + "\n"


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def theta_for(seed, alpha=0.93):
    rng = np.random.default_rng(seed)
    t = np.zeros((3, mj.n_params()))
    t[1, 0] = alpha
    t[2] = rng.normal(0.0, 0.3, mj.n_params())
    return t


def oracle_parts(N, theta, pos):
    spec = SystemSpec(N=N, elements=(SLATER, GAUSSIAN))
    g, lap, pg, en = Oracle().eval(spec, theta[:2, :1], pos)
    J, gJ, lJ = mj.jastrow(theta[2], pos, N, 2)
    return g, lap, en, J, gJ, lJ


@pytest.mark.parametrize("N", [2, 6, 12])
def test_fixed_positions(N):
    from vmachine_b200 import Engine
    theta = theta_for(N)
    rng = np.random.default_rng(100 + N)
    W = 3
    pos = rng.normal(0.0, 1.0, (W, 2 * N))
    # the FP32 network on the CUDA cores throughout (the probe move is a sweep step);
    # the tensor-core sweep is held to this path in test_tensor_core_layer_tracks_fp32
    with Engine(config(N, extra=["mlpTensorCores: false"]), walkers=W, precision=0) as eng:
        eng.set_parameters(theta)
        eng.init_walkers(pos)
        g, lap, pg, en = eng.eval()
        for w in range(W):
            gs, ls, ens, J, gJ, lJ = oracle_parts(N, theta, pos[w])
            assert rel(g[w, 2], gJ) < 2e-5
            assert abs(lap[w, 2] - lJ) < 2e-5 * max(1.0, abs(lJ))
            assert rel(g[w, :2], gs) < 1e-11
            kin = -0.5 * (ls.sum() + lJ + ((gs.sum(0) + gJ) ** 2).sum())
            assert abs(en[w, 0] - kin) < 2e-5 * max(1.0, abs(kin))
            assert rel(en[w, 1:], ens[1:]) < 1e-11
            assert rel(pg[w, 2], mj.param_gradient(theta[2], pos[w], N, 2)) < 1e-4
        # a forced move: the MLP ratio is exp(2 (J(y) - J(x)))
        k = rng.integers(0, 2 * N, W)
        xn = pos[np.arange(W), k] + rng.normal(0.0, 0.3, W)
        r = eng.probe_move(k, xn)
        g2, lap2, pg2, en2 = eng.eval()
        for w in range(W):
            y = pos[w].copy()
            y[k[w]] = xn[w]
            want = np.exp(2.0 * (mj.jastrow_value(theta[2], y, N, 2) -
                                 mj.jastrow_value(theta[2], pos[w], N, 2)))
            assert abs(r[w, 2] - want) < 2e-5 * want
            gs, ls, ens, J, gJ, lJ = oracle_parts(N, theta, y)
            assert rel(g2[w, 2], gJ) < 2e-5
            kin = -0.5 * (ls.sum() + lJ + ((gs.sum(0) + gJ) ** 2).sum())
            assert abs(en2[w, 0] - kin) < 2e-5 * max(1.0, abs(kin))


@pytest.mark.parametrize("N", [6, 20])
def test_tensor_core_backward_at_fixed_positions(N):
    """dJ/dtheta from the tensor-core backward (bfloat16 high/low operands, FP32
    accumulation) against the FP64 oracle and the CUDA-core backward, per walker."""
    from vmachine_b200 import Engine
    theta = theta_for(N + 3)
    rng = np.random.default_rng(200 + N)
    W = 6
    pos = rng.normal(0.0, 1.0, (W, 2 * N))
    pg = {}
    for tc in ("false", "true"):
        with Engine(config(N, extra=[f"mlpTensorCores: {tc}"]), walkers=W, precision=0) as eng:
            eng.set_parameters(theta)
            eng.init_walkers(pos)
            pg[tc] = eng.eval()[2][:, 2]
            assert not (eng.status() & 8).any()
    for w in range(W):
        want = mj.param_gradient(theta[2], pos[w], N, 2)
        assert rel(pg["true"][w], want) < 2e-4
        assert rel(pg["true"][w], pg["false"][w]) < 2e-4


def test_sampled_gradient_sums():
    """One iteration: the MLP rows of the gradient sums come from the window's
    snapshots, scaled to the window's sample count; dJ/db3 is the pair count, so its
    sum is pairs x walkers x sampled window steps."""
    from vmachine_b200 import Engine
    N, W = 6, 64
    with Engine(config(N, steps=W * 600), walkers=W, precision=0) as eng:
        eng.set_parameters(theta_for(5))
        eng.init_walkers(None, seed=3)
        info = eng.info
        sums, g, ge = eng.sample(0, info.steps_per_walker + info.burn_in, info.burn_in)
        assert np.all(np.isfinite(g)) and np.all(np.isfinite(ge))
        assert np.abs(g[2]).max() > 0 and np.abs(ge[2]).max() > 0
        bs = info.steps_per_walker // info.batches
        lo, hi = max(1, info.burn_in), min(bs - 1, info.steps_per_walker + info.burn_in - 1)
        n_win = hi - lo + 1
        assert abs(g[2, 4416] - N * (N - 1) / 2 * W * n_win) < 1e-9 * g[2, 4416]



@pytest.mark.parametrize("compat,sampling", [(0, "importanceSampling"), (0, "bruteForce")])
def test_zero_network_equals_pade(compat, sampling):
    """With zero output layers the MLP factor is the cusp term a_s r / (1 + r), the
    Pade-Jastrow at gamma = 1: on the same replayed stream both engines make the same
    accept/reject decisions and record the same energies (the MLP path in FP32).
    Corrected mode only: under compat the Pade ratio skips partners j < p, which the
    MLP factor does not copy."""
    from vmachine_b200 import Engine
    N, W, steps = 6, 4, 400
    rng = np.random.default_rng(9)
    pos = rng.normal(0.0, 1.0, (W, 2 * N))
    stream = np.stack([rng.random((W, steps)),
                       rng.normal(size=(W, steps)) if sampling == "importanceSampling" else rng.random((W, steps)),
                       rng.random((W, steps))], -1)
    th = np.zeros((3, mj.n_params()))
    th[1, 0] = 0.95
    th[2] = mj.xavier(3)  # hidden layers random, output layers zero
    pade = "\n".join(["numParticles: 6", "numDimensions: 2", "hamiltonian: harmonicOscillator",
                      "omega: 1.0", "interactionStyle: coulomb", "waveFunctionElement: slaterDeterminant",
                      "waveFunctionElement: gaussian", "waveFunctionElement: padeJastrow", "basis: hermite",
                      f"sampling: {sampling}", "stepLength: 0.05", "numSteps: 1000"]) + "\n"
    res = []
    for text, theta in ((pade, np.array([[0.0], [0.95], [1.0]])),
                        (config(N, sampling=sampling), th)):
        with Engine(text, walkers=W, precision=0, compat=compat) as eng:
            eng.set_parameters(theta)
            eng.init_walkers(pos)
            res.append(eng.replay(stream))
    (a0, e0), (a1, e1) = res
    assert np.array_equal(a0, a1)
    assert rel(e1, e0) < 2e-5


@pytest.mark.parametrize("N", [6, 20])
def test_tensor_core_layer_tracks_fp32(N):
    """The sweep's second layer on the tensor cores (bfloat16 operands, the values as a
    high and a low part, FP32 accumulation) against the FP32 CUDA-core network on one
    replayed stream: chains that agree for most of the run and energies within 1e-3
    relative while they do."""
    from vmachine_b200 import Engine
    W, steps = 8, 300
    omega = 1.0 if N == 6 else 0.5
    rng = np.random.default_rng(N + 40)
    pos = rng.normal(0.0, 1.0 / np.sqrt(omega), (W, 2 * N))
    stream = np.stack([rng.random((W, steps)), rng.normal(size=(W, steps)), rng.random((W, steps))], -1)
    theta = theta_for(N + 1)
    theta[2] *= 0.5
    res = {}
    for tc in ("false", "true"):
        with Engine(config(N, omega=omega, extra=[f"mlpTensorCores: {tc}"]), walkers=W, precision=0,
                    compat=0) as eng:
            eng.set_parameters(theta)
            eng.init_walkers(pos)
            res[tc] = eng.replay(stream)
            assert not (eng.status() & 8).any()  # no tensor-core wait gave up
    (a32, e32), (atc, etc) = res["false"], res["true"]
    agree = 0
    for w in range(W):
        diff = np.nonzero(a32[w] != atc[w])[0]
        upto = diff[0] if len(diff) else steps
        agree += upto
        el32, eltc = e32[w, :upto].sum(-1), etc[w, :upto].sum(-1)
        assert np.max(np.abs(eltc - el32) / np.abs(el32)) < 1e-3
    assert agree > 0.8 * W * steps


@pytest.mark.parametrize("N", [6, 20])
def test_mlp_dot_sweep_tracks_general_path(N):
    """The MLP Jastrow on the FP32 dot sweep (mixed precision: incremental pair and
    one-body caches, the tensor-core layer with the CTA in lockstep, FP64 rebuilds)
    against the general FP64 path on one replayed stream: the same decisions for most
    of the run and local energies within 1e-3 relative while the chains agree."""
    from vmachine_b200 import Engine
    from vmachine_b200.engine import KERNEL_DOT, KERNEL_GENERAL
    W, steps = 8, 300
    omega = 1.0 if N == 6 else 0.5
    rng = np.random.default_rng(N + 70)
    pos = rng.normal(0.0, 1.0 / np.sqrt(omega), (W, 2 * N))
    stream = np.stack([rng.random((W, steps)), rng.normal(size=(W, steps)), rng.random((W, steps))], -1)
    theta = theta_for(N + 2)
    theta[2] *= 0.5
    res = {}
    for prec, variant in ((0, KERNEL_GENERAL), (1, KERNEL_DOT)):
        with Engine(config(N, omega=omega), walkers=W, precision=prec, compat=0) as eng:
            assert eng.info.kernel_variant == variant
            eng.set_parameters(theta)
            eng.init_walkers(pos)
            res[prec] = eng.replay(stream)
            assert not (eng.status() & 8).any()
    (a64, e64), (a32, e32) = res[0], res[1]
    agree = 0
    for w in range(W):
        diff = np.nonzero(a64[w] != a32[w])[0]
        upto = diff[0] if len(diff) else steps
        agree += upto
        el64, el32 = e64[w, :upto].sum(-1), e32[w, :upto].sum(-1)
        assert np.max(np.abs(el32 - el64) / np.abs(el64)) < 1e-3, w
    assert agree > 0.8 * W * steps


def test_mlp_dot_trains():
    """One short optimisation on the dot sweep: finite energies and gradients, the
    network's rows move, no walker flagged beyond rejected NaN proposals."""
    from vmachine_b200 import Engine
    N, W = 6, 256
    text = config(N, steps=W * 400, extra=["numWalkers: 256", "precision: mixed", "compat: corrected"])
    with Engine(text) as eng:
        eng.init_walkers(None, seed=2)
        t0 = eng.parameters()
        hist = [eng.run_iteration(it) for it in range(5)]
        t1 = eng.parameters()
        assert all(np.isfinite(a.energy) for a in hist)
        assert np.abs(t1[2] - t0[2]).max() > 0
        assert (int(np.bitwise_or.reduce(eng.status())) & ~2) == 0

