"""Mixed precision on the general path: the atoms' compiled form (hydrogen-orbital
Slater determinants x SimpleJastrow, Coulomb, importance sampling) sweeps in FP32,
with the Slater inverse and its contractions kept in FP64, between FP64
re-inversions; it tracks the FP64 engine.

He (Z = 2, one orbital per spin block) and Ne (Z = 10, 1s 2s 2p blocks of 5): the same
walkers, seeds and parameters in both precisions, one sampling pass of 400 steps per
walker.
- The pass energies agree to half the error bar of the walkers' mean energies.
- Walker by walker, on the chains that stayed together (final positions within
  1e-4), the mean local energies agree to 1e-6 relative at the median and 1e-4 at
  the 99th percentile.  Ne has rare samples next to a coalescence (a nucleus or
  another electron) whose FP32 kinetic energy cancels to a few per cent.
- After three ADAM iterations the He parameters agree to 1e-4.  Ne's gradients are
  dominated by those rare samples, so its optimisation paths part.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pass(text):
    from vmachine_b200 import Engine
    with Engine(text) as e:
        e.init_walkers(None, seed=3)
        s, _, _ = e.sample(0, 420, 20)
        return (s.energy / s.n_samples, e.walker_energies(), e.positions(),
                int(np.bitwise_or.reduce(e.status())), e.info.precision)


@pytest.mark.parametrize("Z", [2, 10])
def test_mixed_atom_tracks_fp64(Z):
    from vmachine_b200.batch import atom_text
    W = 2048
    text = atom_text(Z, W, 400, seed=3)
    E64, w64, x64, st64, _ = _pass(text)
    E32, w32, x32, st32, prec = _pass(text.replace("precision: fp64", "precision: mixed"))
    assert prec == 1
    assert st32 == st64  # the same kinds of walker flags in both (2: a NaN acceptance weight)
    err = np.std(w64, ddof=1) / np.sqrt(W)
    same = np.abs(x32 - x64).max(axis=1) < 1e-4
    rel = np.abs(w32 - w64)[same] / np.abs(w64[same])
    print(f"Z={Z}: fp64 {E64:.8f} mixed {E32:.8f} diff {E32 - E64:.2e} error bar {err:.2e}; "
          f"{same.sum()} of {W} chains together; walker relative difference median {np.median(rel):.2e} "
          f"q99 {np.quantile(rel, 0.99):.2e} max {rel.max():.2e}")
    assert abs(E32 - E64) < 0.5 * err
    assert same.sum() >= W - 8
    assert np.median(rel) < 1e-6
    assert np.quantile(rel, 0.99) < 1e-4


def test_mixed_helium_parameters_track_fp64():
    from vmachine_b200 import Engine
    from vmachine_b200.batch import atom_text
    text = atom_text(2, 2048, 400, seed=3)
    theta = {}
    for prec in ("fp64", "mixed"):
        with Engine(text.replace("precision: fp64", f"precision: {prec}")) as e:
            e.init_walkers(None, seed=3)
            hist = [e.run_iteration(i) for i in range(3)]
            theta[prec] = (np.asarray(e.parameters()), [a.energy for a in hist])
    print("He energies", theta["fp64"][1], theta["mixed"][1])
    assert np.allclose(theta["mixed"][0], theta["fp64"][0], rtol=1e-4, atol=1e-6)
    assert np.allclose(theta["mixed"][1], theta["fp64"][1], rtol=1e-6)


def test_mixed_rejects_the_generic_general_path():
    """Mixed precision takes the atom form only; RBM systems stay FP64."""
    from vmachine_b200 import Engine
    from vmachine_b200.engine import VmcError
    text = "\n".join([
        "numParticles: 2", "numDimensions: 2", "hamiltonian: harmonicOscillator", "omega: 1.0",
        "waveFunctionElement: rbmGaussian", "waveFunctionElement: rbmProduct", "numHiddenNodes: 2",
        "sampling: importanceSampling", "stepLength: 0.01", "numSteps: 4000", "numWalkers: 64",
        "precision: mixed"]) + "\n"
    with pytest.raises(VmcError):
        Engine(text)
