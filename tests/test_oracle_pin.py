"""Pin the C oracle (oracle/vmc_oracle.c) to the reference's own outputs, and check it
against properties that need no reference.

The golden vectors in tests/golden/ were produced by the reference's C++ sources
(tests/golden/make_golden.py).  Bar: 1e-11 relative (max-abs over each array,
relative to its max-abs) for FP64 values, identical accept/reject sequences.  The
densities and the driver schedule are restated on the host (oracle/vmc_oracle_host.py)
around the oracle's chains.  The properties: exact energies (the oscillator's and the
hydrogenic closed shells), the variational bound on the interacting pair, the
stationary distribution of each move type, symmetry of the local energy, and
derivatives against difference quotients of the oracle's own ratios.
"""
import os

import numpy as np
import pytest

from oracle_bind import GAUSSIAN, PADE, SLATER, Oracle, SystemSpec, load_cases, spec_from_case

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden")
TOL = 1e-11

ORACLE = None


def oracle():
    global ORACLE
    if ORACLE is None:
        ORACLE = Oracle()
    return ORACLE


def rel(a, b):
    a, b = np.asarray(a, np.float64), np.asarray(b, np.float64)
    scale = max(np.max(np.abs(b)) if b.size else 0.0, 1e-300)
    return float(np.max(np.abs(a - b)) / scale) if b.size else 0.0


EVAL = load_cases(os.path.join(GOLD, "eval_fixed.npz"))
CHAINS = load_cases(os.path.join(GOLD, "chains.npz"))
ITERS = load_cases(os.path.join(GOLD, "iterations.npz"))
BLOCK = load_cases(os.path.join(GOLD, "blocking.npz"))
# Slater determinants of hydrogen orbitals (He, Be, Ne, Mg, Ar): fixed positions and chains
for _f in ("hydrogen_orbitals.npz", "hydrogen_simplejastrow.npz"):
    _H = load_cases(os.path.join(GOLD, _f))
    EVAL.update({k: v for k, v in _H.items() if not k.startswith("chain_")})
    CHAINS.update({k[len("chain_"):]: v for k, v in _H.items() if k.startswith("chain_")})


@pytest.mark.parametrize("name", sorted(EVAL))
def test_fixed_positions(name):
    c = EVAL[name]
    spec = spec_from_case(c)
    O = oracle()
    for t in range(len(c["pos"])):
        pos = c["pos"][t]
        g, lap, pg, en = O.eval(spec, c["theta"], pos)
        assert rel(g, c["grad"][t]) < TOL
        assert rel(lap, c["lap"][t]) < TOL
        assert rel(pg, c["pgrad"][t]) < TOL
        assert rel(en, c["energies"][t]) < TOL
        k, xn = int(c["k"][t]), float(c["xnew"][t])
        r = O.ratio(spec, c["theta"], pos, k, xn)
        assert rel(r, c["ratios"][t]) < TOL
        pos2 = pos.copy()
        pos2[k] = xn
        g, lap, pg, en = O.eval(spec, c["theta"], pos2)
        assert rel(g, c["grad2"][t]) < TOL
        assert rel(lap, c["lap2"][t]) < TOL
        assert rel(pg, c["pgrad2"][t]) < TOL
        assert rel(en, c["energies2"][t]) < TOL


@pytest.mark.parametrize("name", sorted(CHAINS))
def test_replayed_chain(name):
    c = CHAINS[name]
    spec = spec_from_case(c)
    O = oracle()
    steps = len(c["accepted"])
    pos = c["pos"][None].copy()
    f = O.quantum_force(spec, c["theta"], c["pos"])[None].copy()
    out = O.run(spec, c["theta"], pos, f, steps, 0, 0, 1, stream=c["stream"][None])
    assert np.array_equal(out["accepted"][0], c["accepted"])
    assert rel(out["energies"][0], c["energies"]) < TOL
    assert rel(pos[0], c["final_pos"]) < TOL


def _run_iterations(c, spec, O):
    from oracle.vmc_oracle_host import Adam, GradientDescent, averages, energy_gradient
    theta = c["theta0"].copy()
    E, P = theta.shape
    burn, steps_wo, batches = int(c["burn_in"]), int(c["steps_wo"]), int(c["batches"])
    per = burn + steps_wo
    opt = spec.optimization.split()
    if opt[0] == "adam":
        optim = Adam(theta.shape, spec.learning_rate)
    else:
        gamma, power = (float(opt[1]), float(opt[2])) if len(opt) >= 3 else (0.0, 0.0)
        optim = GradientDescent(theta.shape, spec.learning_rate, gamma, power)
    assert optim.batches == batches
    pos = c["pos"][None].copy()
    f = O.quantum_force(spec, theta, c["pos"])[None].copy()
    # Pade pair terms keep the gamma they were computed with until their particle moves
    gpair = np.zeros((1, spec.N, spec.N))
    if 2 in spec.elements:
        gpair[:] = theta[list(spec.elements).index(2), 0]
    res = []
    for it in range(len(c["energy"])):
        stream = c["stream"][it * per:(it + 1) * per][None]
        out = O.run(spec, theta, pos, f, per, burn, it, batches, stream=stream, want_steps=False,
                    gpair=gpair)
        avg = averages(out["sums"].sum(0), steps_wo, steps_wo // batches, (E, P))
        theta = theta - optim.update(energy_gradient(avg))
        res.append((avg, theta.copy()))
    return res


@pytest.mark.parametrize("name", sorted(ITERS))
def test_iterations(name):
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    c = ITERS[name]
    spec = spec_from_case(c)
    res = _run_iterations(c, spec, oracle())
    for it, (avg, theta) in enumerate(res):
        for key in ("energy", "kinetic", "external", "interaction", "acceptance"):
            assert rel(avg[key], c[key][it]) < TOL, (key, it)
        assert rel(avg["std_error"], c["std_error"][it]) < 1e-8
        assert rel(avg["avg_grad"], c["avg_grad"][it]) < TOL
        assert rel(avg["avg_grad_e"], c["avg_grad_e"][it]) < TOL
        assert rel(theta, c["params"][it]) < TOL


@pytest.mark.parametrize("name", sorted(BLOCK))
def test_blocking(name):
    c = BLOCK[name]
    mean, var = oracle().blocking(c["x"])
    assert abs(mean - float(c["mean"])) < 1e-12 * max(1.0, abs(float(c["mean"])))
    assert abs(np.sqrt(var) - float(c["std_error"])) < 1e-9 * float(c["std_error"])


def test_drift_limiter_in_the_oracle():
    """The corrected mode's drift limiter in the oracle (driftLimit: a): a tiny a leaves
    a replayed chain as it is without the limiter, a = 0.5 changes it, and the
    reference mode ignores the constant (its proposal is the reference's)."""
    spec0 = SystemSpec(N=6, elements=(SLATER, GAUSSIAN, PADE), step=0.05, quirks=0)
    rng = np.random.default_rng(3)
    steps = 200
    pos = rng.normal(size=(1, spec0.D))
    stream = np.stack([rng.random(steps), rng.normal(size=steps), rng.random(steps)], -1)[None]
    theta = np.array([[0.0], [0.95], [0.6]])
    O = Oracle()

    def chain(spec):
        p = pos.copy()
        return O.run(spec, theta, p, np.zeros_like(p), steps, 0, 0, 1, stream=stream), p

    (base, p0) = chain(spec0)
    tiny, p1 = chain(SystemSpec(N=6, elements=(SLATER, GAUSSIAN, PADE), step=0.05, quirks=0, drift_limit=1e-12))
    assert np.array_equal(base["accepted"], tiny["accepted"])
    assert np.allclose(p0, p1, rtol=1e-9, atol=1e-12)
    lim, p2 = chain(SystemSpec(N=6, elements=(SLATER, GAUSSIAN, PADE), step=0.05, quirks=0, drift_limit=0.5))
    assert not np.allclose(p0, p2)
    ref0, r0 = chain(SystemSpec(N=6, elements=(SLATER, GAUSSIAN, PADE), step=0.05))
    ref1, r1 = chain(SystemSpec(N=6, elements=(SLATER, GAUSSIAN, PADE), step=0.05, drift_limit=0.5))
    assert np.array_equal(ref0["accepted"], ref1["accepted"]) and np.array_equal(r0, r1)


DENS = load_cases(os.path.join(GOLD, "densities.npz"))
SCHED = load_cases(os.path.join(GOLD, "schedules.npz"))


@pytest.mark.parametrize("name", sorted(DENS))
def test_densities(name):
    """The oracle's chains, binned after every step by the host restatement of the
    Sampler's densities, give exactly the reference's counts (tests/golden/densities.npz:
    its own Sampler on the same replayed numbers, summed over walkers).  An atom's
    densities see the current radii; a dot's radial densities the starting ones."""
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    from oracle.vmc_oracle_host import DensityCounts, radial_vector_updated, radii
    from oracle_bind import HYDROGENLIKE
    c = DENS[name]
    spec = spec_from_case(c)
    O = oracle()
    counts = DensityCounts(int(c["bins"]), float(c["max_radius"]))
    moving = radial_vector_updated(spec.atom, HYDROGENLIKE in spec.elements)
    W, steps = c["stream"].shape[:2]
    for w in range(W):
        pos = c["pos"][w][None].copy()
        f = O.quantum_force(spec, c["theta"], c["pos"][w])[None].copy()
        r0 = radii(pos[0], spec.d)
        for s in range(steps):
            O.run(spec, c["theta"], pos, f, 1, 0, 0, 1, stream=c["stream"][w:w + 1, s:s + 1], want_steps=False)
            counts.add(pos[0], radii(pos[0], spec.d) if moving else r0, spec.d)
    assert np.array_equal(counts.spatial, c["spatial"])
    assert np.array_equal(counts.radial, c["radial"])
    assert np.array_equal(counts.pair, c["pair"])


@pytest.mark.parametrize("name", sorted(SCHED))
def test_simulation_schedule(name):
    """System::runSimulation's schedule (convergence check, adaptive steps) restated on
    the host around the oracle's iterations gives the reference's step counts, density
    iteration and energies on the same replayed numbers (tests/golden/schedules.npz)."""
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    from oracle.vmc_oracle_host import Adam, Schedule, averages, energy_gradient
    c = SCHED[name]
    spec = spec_from_case(c)
    keys = dict(line.split(": ", 1) for line in str(c["extra"]).split("\n") if line)
    on = {"true": True, "false": False}
    sched = Schedule(int(keys["numIterations"]), spec.num_steps,
                     adaptive=on[keys["applyAdaptiveSteps"]], range_=int(keys["rangeOfAdaptiveSteps"]),
                     additional=int(keys["additionalSteps"]), additional_last=int(keys["additionalStepsLastIter"]),
                     check=on[keys["checkConvergence"]], n_energies=int(keys["numberOfEnergies"]),
                     tolerance=float(keys["tolerance"]))
    assert spec.optimization == "adam" and spec.sampling == "bruteForce"
    O = oracle()
    theta = c["theta"].copy()
    E, P = theta.shape
    optim = Adam(theta.shape, spec.learning_rate)
    pos = c["pos"][None].copy()
    f = np.zeros_like(pos)
    gpair = np.zeros((1, spec.N, spec.N))
    if PADE in spec.elements:
        gpair[:] = theta[list(spec.elements).index(PADE), 0]
    # burn-in: the equilibration fraction main() sets, 0.001 (main.cpp:10), of the
    # initial step count, the same in every iteration (userinput.cpp:74)
    burn = int(spec.num_steps * 0.001)
    off, steps, energy, last = 0, [], [], []
    for it in range(sched.n_iterations):
        n = sched.steps(it)
        stream = c["stream"][off:off + n + burn][None]
        off += n + burn
        out = O.run(spec, theta, pos, f, n + burn, burn, it, optim.batches, stream=stream, want_steps=False,
                    gpair=gpair)
        avg = averages(out["sums"].sum(0), n, n // optim.batches, (E, P))
        theta = theta - optim.update(energy_gradient(avg))
        steps.append(n)
        last.append(int(sched.is_density_iteration(it)))
        energy.append(avg["energy"])
        sched.after(it, avg["energy"])
    assert steps == [int(v) for v in c["steps"]]
    assert last == [int(v) for v in c["last"]]
    assert rel(energy, c["energy"]) < TOL


def test_exact_energies():
    """The exact ground states the reference's tests use: two non-interacting
    electrons in the 2D oscillator, omega = 1, with the Gaussian at alpha = 1, have
    E_L = 2 at every position (zero variance); a Slater determinant of Hermite
    orbitals times that Gaussian is the exact closed-shell state of N = 6 and 12,
    E_L = sum of the shell energies (10 and 28) everywhere; and the same holds for
    hydrogen-orbital determinants of atoms without the repulsion."""
    O = oracle()
    rng = np.random.default_rng(5)
    for N, exact, elements in ((2, 2.0, (GAUSSIAN,)), (6, 10.0, (SLATER, GAUSSIAN)),
                               (12, 28.0, (SLATER, GAUSSIAN))):
        spec = SystemSpec(N=N, elements=elements, coulomb=False, omega=1.0)
        theta = np.zeros((len(elements), spec.p_max))
        theta[list(elements).index(GAUSSIAN), 0] = 1.0
        for _ in range(5):
            _, _, _, en = O.eval(spec, theta, rng.normal(0.0, 1.0, spec.D))
            assert abs(en.sum() - exact) < 1e-10 * exact, (N, en)
            assert en[2] == 0.0
    # hydrogenic atoms without the electrons' repulsion: a Slater determinant of
    # hydrogen orbitals is exact, E_L = -sum Z^2 / (2 n^2) everywhere (He 1s^2,
    # Be 1s^2 2s^2, Ne 1s^2 2s^2 2p^6)
    for N, Z, exact in ((2, 2, -4.0), (4, 4, -20.0), (10, 10, -200.0)):
        spec = SystemSpec(N=N, Z=Z, d=3, elements=(SLATER,), atom=True, basis="hydrogenOrbital",
                          coulomb=False)
        theta = np.zeros((1, max(spec.p_max, 1)))
        for _ in range(5):
            _, _, _, en = O.eval(spec, theta, rng.normal(0.0, 1.0, spec.D))
            assert abs(en.sum() - exact) < 1e-12 * abs(exact), (N, en)


def test_interacting_pair_optimises_toward_exact():
    """The reference's CPU-runnable case, shortened: two interacting electrons in the
    2D oscillator (omega = 1, Coulomb), Gaussian (alpha 1.0) x Pade (beta 0.5),
    brute-force moves of stepLength 0.1 from uniform starts in [-1, 1]^2, gradient
    descent at lr 0.1, 40 iterations of 10^5 steps in the oracle.  The exact energy is
    3 a.u.: every iteration's energy lies above it up to 5 blocked error bars
    (variational principle), the optimisation lowers it, and it ends within 0.01."""
    import sys
    sys.path.insert(0, os.path.dirname(HERE))
    from oracle.vmc_oracle_host import GradientDescent, averages, energy_gradient
    O = oracle()
    spec = SystemSpec(N=2, elements=(GAUSSIAN, PADE), sampling="bruteForce", step=0.1,
                      optimization="gradientDescent", learning_rate=0.1)
    theta = np.zeros((2, spec.p_max))
    theta[0, 0], theta[1, 0] = 1.0, 0.5
    pos = np.random.default_rng(3).uniform(-1.0, 1.0, (1, spec.D))
    f = np.zeros_like(pos)
    opt = GradientDescent(theta.shape, 0.1)
    counter = np.zeros(1, np.uint64)
    steps, burn = 100000, 100
    energies = []
    for it in range(40):
        out = O.run(spec, theta, pos, f, steps + burn, burn, it, opt.batches, seed=7, counter=counter)
        avg = averages(out["sums"].sum(0), steps, steps // opt.batches, theta.shape)
        series = out["energies"][0, burn:burn + 65536].sum(axis=1)
        _, var = O.blocking(series)
        assert avg["energy"] > 3.0 - 5.0 * np.sqrt(var), (it, avg["energy"], np.sqrt(var))
        energies.append(avg["energy"])
        theta = theta - opt.update(energy_gradient(avg))
    assert energies[0] - energies[-1] > 0.01
    assert abs(energies[-1] - 3.0) < 0.01


def test_importance_sampling_stationary_distribution():
    """Detailed balance of the oracle's importance sampling, measured: two
    non-interacting electrons in the 2D oscillator (omega = 1) under a Gaussian of
    alpha = 0.8 have <E_L> = alpha + 1/alpha exactly when the chain samples |Psi|^2.
    32 chains of 38 000 steps at dt = 0.2:
    - the corrected Fokker-Planck Green's ratio samples it (within 4 error bars), and so
      does the drift-limited form (driftLimit 0.5: limited drift in the proposal and in
      the ratio);
    - the reference's Green's ratio (importancesampling.cpp:43-47, reproduced under
      compat: reference) does not: its chains sit more than 20 error bars low, the
      bias that compat: corrected removes;
    - brute-force moves (bruteforce.cpp:26-52, stepLength 0.2) sample it."""
    from oracle_bind import Q_ALL
    O = oracle()
    alpha = 0.8
    exact = alpha + 1.0 / alpha
    W, steps, burn = 32, 40000, 2000
    theta = np.array([[alpha]])
    res = {}
    for name, quirks, a in (("corrected", 0, 0.0), ("limited", 0, 0.5), ("reference", Q_ALL, 0.0),
                            ("brute force", Q_ALL, 0.0)):
        sampling = "bruteForce" if name == "brute force" else "importanceSampling"
        spec = SystemSpec(N=2, elements=(GAUSSIAN,), coulomb=False, omega=1.0,
                          sampling=sampling, step=0.2, quirks=quirks, drift_limit=a)
        pos = np.random.default_rng(2).normal(0.0, 1.0, (W, spec.D))
        f = np.stack([O.quantum_force(spec, theta, p) for p in pos])
        out = O.run(spec, theta, pos, f, steps, burn, 0, 1, seed=11, counter=np.zeros(W, np.uint64),
                    want_steps=False)
        means = out["sums"][:, 0] / (steps - burn)
        res[name] = (means.mean(), means.std(ddof=1) / np.sqrt(W))
    for name in ("corrected", "limited", "brute force"):
        e, err = res[name]
        assert abs(e - exact) < 4 * err, (name, e, err)
    e, err = res["reference"]
    assert exact - e > 20 * err, res


def test_local_energy_symmetries():
    """|Psi|^2 of a closed-shell dot (Slater determinant of Hermite orbitals x Gaussian x
    Pade) is unchanged by exchanging two electrons of the same spin and by rotating all
    positions about the origin (the closed shells fill every orbital of a degenerate
    level), so the oracle's local-energy parts are too."""
    O = oracle()
    rng = np.random.default_rng(12)
    for N in (6, 12):
        spec = SystemSpec(N=N, elements=(SLATER, GAUSSIAN, PADE), omega=1.0)
        theta = np.zeros((3, spec.p_max))
        theta[1, 0], theta[2, 0] = 0.9, 0.4
        x = rng.normal(0.0, 1.0, (N, 2))
        en = O.eval(spec, theta, x.ravel())[3]
        h = N // 2
        for a, b in ((0, 2), (h, h + 1)):
            y = x.copy()
            y[[a, b]] = y[[b, a]]
            assert rel(O.eval(spec, theta, y.ravel())[3], en) < 1e-11
        c, s = np.cos(0.7), np.sin(0.7)
        rot = x @ np.array([[c, -s], [s, c]]).T
        assert rel(O.eval(spec, theta, rot.ravel())[3], en) < 1e-10


@pytest.mark.parametrize("case", ["dot6", "he_sj", "rbm"])
def test_derivatives_consistent_with_ratios(case):
    """Each element's gradient and Laplacian of ln Psi equal the central differences
    of the log of its own |Psi|^2 ratio for single-coordinate moves (corrected mode),
    and T = -1/2 (lap + |grad|^2) follows.  The one exception is the reference's own:
    RBMGaussian's ratio is exp(((x_old - a)^2 - (x_new - a)^2) / (2 sigma^2))
    (rbmgaussian.cpp:43-45), the ratio of the amplitudes, while its gradient
    -(x - a) / sigma^2 and Laplacian belong to the same Gaussian (RBMProduct squares
    its ratio, rbmproduct.cpp:115); so the difference quotients give half of them, and
    a chain with RBMGaussian samples |Psi_G| |Psi_rest|^2."""
    from oracle_bind import RBMGAUSSIAN, RBMPRODUCT, SIMPLEJASTROW
    spec = {"dot6": SystemSpec(N=6, elements=(SLATER, GAUSSIAN, PADE), omega=1.0, quirks=0),
            "he_sj": SystemSpec(N=2, Z=2, d=3, elements=(SLATER, SIMPLEJASTROW), atom=True,
                                basis="hydrogenOrbital", quirks=0),
            "rbm": SystemSpec(N=2, elements=(RBMGAUSSIAN, RBMPRODUCT), hidden=2, quirks=0)}[case]
    O = oracle()
    rng = np.random.default_rng(3)
    theta = rng.normal(0.5, 0.1, (len(spec.elements), spec.p_max))
    x = rng.normal(0.0, 1.0, spec.D)
    g, lap, _, en = O.eval(spec, theta, x)
    h = 1e-4
    gfd, d2 = np.zeros_like(g), np.zeros(len(spec.elements))
    for k in range(spec.D):
        rp = np.log(O.ratio(spec, theta, x, k, x[k] + h))
        rm = np.log(O.ratio(spec, theta, x, k, x[k] - h))
        gfd[:, k] = (rp - rm) / (4 * h)
        d2 += (rp + rm) / (2 * h * h)
    half = np.array([0.5 if e == RBMGAUSSIAN else 1.0 for e in spec.elements])
    assert rel(gfd, g * half[:, None]) < 1e-6
    assert rel(d2, lap * half) < 1e-6
    if RBMGAUSSIAN not in spec.elements:
        G = g.sum(0)
        assert abs(-0.5 * (d2.sum() + G @ G) - en[0]) < 1e-6 * max(1.0, abs(en[0]))


@pytest.mark.parametrize("case", ["dot6", "he_sj", "rbm"])
def test_parameter_gradients_consistent_with_ratios(case):
    """d ln(ratio) / d theta for a fixed move equals 2 (dlnPsi/dtheta at the new point
    minus at the old) for every parameter (corrected mode), up to two of the
    reference's own factors, both reproduced: RBMGaussian's amplitude ratio (1 instead
    of 2, rbmgaussian.cpp:43-45), and RBMProduct's weight gradient x n, which lacks the
    1 / sigma^2 its ratio carries (rbmproduct.cpp:95-101 against :106, with
    sigma = 10 x the width, :15): the reference's ADAM sees the weights' gradient
    sigma^2 = 100 / omega times too large."""
    from oracle_bind import RBMGAUSSIAN, RBMPRODUCT, SIMPLEJASTROW
    spec = {"dot6": SystemSpec(N=6, elements=(SLATER, GAUSSIAN, PADE), omega=1.0, quirks=0),
            "he_sj": SystemSpec(N=2, Z=2, d=3, elements=(SLATER, SIMPLEJASTROW), atom=True,
                                basis="hydrogenOrbital", quirks=0),
            "rbm": SystemSpec(N=2, elements=(RBMGAUSSIAN, RBMPRODUCT), hidden=2, quirks=0)}[case]
    O = oracle()
    rng = np.random.default_rng(5)
    theta = rng.normal(0.5, 0.1, (len(spec.elements), spec.p_max))
    x = rng.normal(0.0, 1.0, spec.D)
    k, xn = 1, x[1] + 0.3
    x2 = x.copy()
    x2[k] = xn
    dpg = O.eval(spec, theta, x2)[2] - O.eval(spec, theta, x)[2]
    sigma2 = (10.0 / np.sqrt(spec.omega)) ** 2
    h = 1e-6
    for e, el in enumerate(spec.elements):
        for p in range(spec.n_params(e)):
            tp, tm = theta.copy(), theta.copy()
            tp[e, p] += h
            tm[e, p] -= h
            d = (np.log(O.ratio(spec, tp, x, k, xn)[e]) - np.log(O.ratio(spec, tm, x, k, xn)[e])) / (2 * h)
            want = 2.0 * dpg[e, p]
            if el == RBMGAUSSIAN:
                want = dpg[e, p]
            elif el == RBMPRODUCT and p >= spec.hidden:
                want /= sigma2
            assert abs(d - want) < 1e-6 * max(1e-2, abs(want)), (el, p, d, want)
