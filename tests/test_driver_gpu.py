"""The reference's driver around the iterations (System::runSimulation,
system.cpp:81-139) and its electron densities (sampler.cpp:639-692), on the GPU.

- vmc_densities counts, step by step, exactly the bins a host computes from the
  walkers' positions after each step (FP64 engine; the binning restated here from
  sampler.cpp:639-692), and on replayed random numbers exactly the counts the
  reference's own Sampler makes along the same chains (tests/golden/densities.npz:
  He and Be on hydrogen orbitals, all three densities; a dot, the spatial density:
  the reference never updates a dot's radial vector, elementoperation.cpp:130-170,
  so its radial densities count the starting radii, where the engine counts the
  current ones);
- vmc_run_simulation: the convergence check ends the run rangeOfAdaptiveSteps + 1
  iterations after convergence, adaptive steps lengthen the last iterations, the
  energy files get one line per iteration, the last iteration writes the density
  files, blocks its energies and writes them to the instant-energy file
  (doResampling)."""
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

DOT6 = ["numParticles: 6", "numDimensions: 2", "hamiltonian: harmonicOscillator", "omega: 0.8",
        "interactionStyle: coulomb", "waveFunctionElement: slaterDeterminant", "waveFunctionElement: gaussian",
        "waveFunctionElement: padeJastrow", "basis: hermite", "sampling: importanceSampling", "stepLength: 0.05",
        "optimization: adam", "learningRate: 0.01", "precision: fp64"]


def text(walkers, steps_per_walker, extra=()):
    return "\n".join(DOT6 + [f"numWalkers: {walkers}", f"numSteps: {walkers * steps_per_walker}"] + list(extra)) + "\n"


def host_bins(pos, N, bins, max_radius):
    step = max_radius / bins
    half = bins // 2
    radial = np.zeros(bins, np.int64)
    grid = np.zeros((bins, bins), np.int64)
    pair = np.zeros((bins, bins), np.int64)
    for p in pos:
        x = p.reshape(N, 2)
        r = np.sqrt(x[:, 0] * x[:, 0] + x[:, 1] * x[:, 1])
        for i in range(N):
            if r[i] < max_radius and int(r[i] / step) < bins:
                radial[int(r[i] / step)] += 1
            ix, iy = int(x[i, 0] / (2 * step)), int(x[i, 1] / (2 * step))
            if abs(ix) < half and abs(iy) < half:
                grid[iy + half, ix + half] += 1
        for i in range(N):
            bi = int(r[i] / step) + 1
            for j in range(i + 1, N):
                bj = int(r[j] / step) + 1
                if bi < bins and bj < bins:
                    pair[bi, bj] += 1
    return radial, grid, pair


DENS = None


def density_cases():
    global DENS
    if DENS is None:
        from oracle_bind import load_cases
        DENS = load_cases(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "densities.npz"))
    return DENS


@pytest.mark.parametrize("name", ["he_horb_sj", "be_horb_pade", "n6_slater_gauss_pade"])
def test_densities_match_reference_sampler(name):
    from oracle_bind import spec_from_case
    from vmachine_b200 import Engine
    c = density_cases()[name]
    spec = spec_from_case(c)
    pos, stream = c["pos"], c["stream"]
    W, steps = pos.shape[0], stream.shape[1]
    bins, rmax = int(c["bins"]), float(c["max_radius"])
    with Engine(spec.input_in(), walkers=W, precision=0, compat=1) as e:
        e.set_parameters(c["theta"])
        e.init_walkers(pos)
        e.set_replay(stream)
        r, sp, tb = e.densities(steps, 0, bins, rmax, radial=True, spatial=True, two_body=True)
    assert np.array_equal(sp.astype(np.int64), c["spatial"])
    if spec.atom:
        assert np.array_equal(r.astype(np.int64), c["radial"])
        assert np.array_equal(tb.astype(np.int64), c["pair"])
    else:
        # the same number of counts, binned at the current radii
        assert r.sum() <= c["radial"].sum() and tb.sum() > 0


@pytest.mark.parametrize("name", ["n2_converge", "n2_no_converge"])
def test_simulation_schedule_matches_reference(name):
    """vmc_run_simulation on one walker against the reference's own System::runSimulation
    loop (tests/golden/schedules.npz: adaptiveSteps, checkingConvergence) on the same
    replayed numbers: the same iterations with the same step counts, so the same
    energies, including the iterations after the density iteration that the
    reference's loop still runs."""
    from oracle_bind import load_cases, spec_from_case
    from vmachine_b200 import Engine
    c = load_cases(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "schedules.npz"))[name]
    spec = spec_from_case(c)
    spec.extra = str(c["extra"]).split("\n")
    with Engine(spec.input_in(), walkers=1, precision=0, compat=1) as e:
        e.set_parameters(c["theta"])
        e.init_walkers(c["pos"][None, :])
        e.set_replay(c["stream"][None, :, :])
        hist = e.run_simulation()
    energy = np.array([a.energy for a in hist])
    assert len(energy) == len(c["energy"])
    assert np.allclose(energy, c["energy"], rtol=1e-10, atol=0), np.abs(energy - c["energy"]).max()


def test_densities_match_host_binning():
    from vmachine_b200 import Engine
    N, W, bins, rmax = 6, 32, 40, 3.0
    with Engine(text(W, 100)) as e:
        e.init_walkers(None, seed=4)
        tot = [np.zeros(bins, np.int64), np.zeros((bins, bins), np.int64), np.zeros((bins, bins), np.int64)]
        dev = [np.zeros(bins, np.int64), np.zeros((bins, bins), np.int64), np.zeros((bins, bins), np.int64)]
        for _ in range(40):
            r, sp, tb = e.densities(1, 0, bins, rmax, radial=True, spatial=True, two_body=True)
            h = host_bins(e.positions(), N, bins, rmax)
            for q in range(3):
                tot[q] += h[q]
            dev[0] += r.astype(np.int64)
            dev[1] += sp.astype(np.int64)
            dev[2] += tb.astype(np.int64)
    for q in range(3):
        assert np.array_equal(dev[q], tot[q]), q
    assert tot[0].sum() > 0.9 * 40 * W * N and tot[2].sum() > 0


def test_run_simulation_driver(tmp_path):
    from vmachine_b200 import Engine
    W, spw, bins = 64, 512, 50
    extra = ["numIterations: 6", "rangeOfAdaptiveSteps: 2", "applyAdaptiveSteps: true", "additionalSteps: 1",
             "additionalStepsLastIter: 2", "printEnergyToFile: true", "computeOneBodyDensity: true",
             "computeOneBodyDensity2: true", "numberOfBins: 50", "maxRadius: 4.0", "doResampling: true",
             f"path: {tmp_path}/"]
    with Engine(text(W, spw, extra)) as e:
        e.init_walkers(None, seed=3)
        hist = e.run_simulation()
        assert len(hist) == 6
        blk = e.last_blocking()
        burn = e.info.burn_in
    # the last iteration samples 2^2 x the steps
    assert blk.samples_per_walker == 1 << int(np.log2(4 * spw))
    assert blk.energy.mean > 0 and blk.energy.std_error > 0 and blk.energy_walkers.std_error > 0
    for f in ("energy.dat", "kinetic.dat", "external.dat", "interaction.dat"):
        vals = np.loadtxt(tmp_path / f)
        assert vals.shape == (6,)
    assert np.allclose(np.loadtxt(tmp_path / "energy.dat"), [a.energy for a in hist], rtol=1e-5)
    one = np.loadtxt(tmp_path / "onebody.dat")
    assert one.shape == (bins,) and 0.9 * W * 4 * spw * 6 < one.sum() <= W * 4 * spw * 6
    grid = np.loadtxt(tmp_path / "onebody2.dat")
    assert grid.shape == (bins, bins) and grid.sum() > 0
    inst = np.loadtxt(tmp_path / "0_0.dat")  # the last iteration's E_L, walker after walker
    assert inst.shape == (W * 4 * spw,)
    assert abs(inst.mean() - hist[-1].energy) < 1e-4 * abs(hist[-1].energy)
    del burn


@pytest.mark.parametrize("tol,compat,expect", [(1e9, "corrected", 4), (1e9, "reference", 6),
                                               (1e-30, "corrected", 6), (1e-30, "reference", 6)])
def test_convergence_check(tol, compat, expect):
    """numberOfEnergies 5, rangeOfAdaptiveSteps 2: with a huge tolerance the run
    converges at iteration 0, so its density iteration is 0 + 1 + 2; the corrected
    driver ends there, the reference's loop runs on to numIterations (the schedule
    itself is held to the reference's in test_simulation_schedule_matches_reference);
    with no tolerance it runs all 6."""
    from vmachine_b200 import Engine
    extra = ["numIterations: 6", "rangeOfAdaptiveSteps: 2", "checkConvergence: true", f"tolerance: {tol!r}",
             "numberOfEnergies: 5", f"compat: {compat}"]
    with Engine(text(32, 200, extra)) as e:
        e.init_walkers(None, seed=1)
        assert len(e.run_simulation()) == expect


def test_nan_energy_average_takes_no_step():
    """A pass whose energy average is NaN while its kinetic average is finite (a NaN
    from the potential alone) returns VMC_E_NAN and leaves the parameters as they
    were; the same pass with its genuine totals then takes the step."""
    from vmachine_b200 import Engine
    from vmachine_b200.engine import Sums, VmcError
    with Engine(text(16, 100)) as e:
        e.init_walkers(None, seed=1)
        s, g, ge = e.sample(0, 200, 20)
        before = e.parameters().copy()
        bad = Sums.from_buffer_copy(s)
        bad.energy = float("nan")
        with pytest.raises(VmcError) as err:
            e.apply_sums(bad, g, ge)
        assert err.value.code == -5
        assert np.array_equal(e.parameters(), before)
        a = e.apply_sums(s, g, ge)
        assert np.isfinite(a.energy) and not np.array_equal(e.parameters(), before)
