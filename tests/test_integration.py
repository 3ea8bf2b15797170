"""The reference-side adapter (integration/b200engine.{h,cpp}, integration/b200_vmc.cpp).

A VMaChine build compiles and links against include/vmc_b200.h and libvmc_b200.so: the
adapter is compiled with the reference's own headers and linked with the reference's
compiled sources (oracle/_ref/libvmref.so).  On the GPU, the driver's engine mode
(B200Engine + the B200Optimization stand-in) gives the same iterations as the Python
binding of the same C ABI, and the reference's own System::runSimulation with its
Metropolis replaced by B200Metropolis prints the same iterations as the reference
program with its own Metropolis on the same random numbers.
"""
import json
import os
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REFDIR = os.environ.get("VMC_REFERENCE_DIR", "/root/reference")
BIN = os.path.join(ROOT, "integration", "_build", "b200_vmc")

# a dot in the reference's key schema only (its parser rejects other keys); no
# `sampling:` key, so the driver's Metropolis stays in place (parser.cpp:210-222)
DOT = """numParticles: 6
numDimensions: 2
hamiltonian: harmonicOscillator
omega: 1.0
interactionStyle: coulomb
waveFunctionElement: slaterDeterminant
waveFunctionElement: gaussian
waveFunctionElement: padeJastrow
basis: hermite
stepLength: 0.05
optimization: adam
learningRate: 0.01
numSteps: {steps}
numIterations: 3
rng: MersenneTwister 17
path: {path}/
"""


def iteration_lines(out):
    """The reference's terminal results (System::printToTerminal): the per-iteration
    lines (step, energy, STD, kinetic, STD, external, STD, interaction, STD, acceptance,
    CPU time; the CPU time dropped) of every iteration but the last, then the last
    iteration's summary values (energies with their STD, acceptance)."""
    rows, final = [], []
    for ln in out.splitlines():
        f = ln.split()
        if len(f) == 11 and f[0].isdigit():
            rows.append([float(x) for x in f[:10]])
        elif ":" in ln and ("energy" in ln.lower() or "Acceptence" in ln) and "Print" not in ln:
            final += [float(t.strip("()")) for t in ln.split(":", 1)[1].replace("=", " ").split()
                      if t.strip("()").replace(".", "", 1).replace("-", "", 1).isdigit()]
    return np.array(rows), np.array(final)


def test_adapter_builds_against_reference():
    if not os.path.isdir(os.path.join(REFDIR, "src")):
        pytest.skip("the reference sources are not on this machine")
    if not os.path.exists(os.path.join(ROOT, "oracle", "_ref", "libvmref.so")):
        subprocess.run(["make", "-C", os.path.join(ROOT, "oracle"), "-j8", "ref", f"REFDIR={REFDIR}"], check=True,
                       capture_output=True)
    if not os.path.exists(os.path.join(ROOT, "vmachine_b200", "libvmc_b200.so")):
        pytest.skip("libvmc_b200.so is not built")
    r = subprocess.run(["make", "-C", os.path.join(ROOT, "integration"), f"REFDIR={REFDIR}"], capture_output=True,
                       text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    assert os.path.exists(BIN)


def test_adapter_runs_the_reference_loop_on_cpu(tmp_path):
    """The driver's reference mode is the reference program: it needs no GPU."""
    if not os.path.exists(BIN):
        pytest.skip("integration/_build/b200_vmc is not built (needs the reference sources)")
    cfg = tmp_path / "input.in"
    cfg.write_text(DOT.format(steps=3000, path=tmp_path))
    r = subprocess.run([BIN, str(cfg), "reference"], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    rows, final = iteration_lines(r.stdout)
    assert rows.shape == (2, 10) and np.all(np.isfinite(rows)) and len(final) == 9


@pytest.mark.gpu
def test_adapter_engine_mode_matches_binding(tmp_path):
    """B200Engine + B200Optimization through the driver against vmachine_b200.Engine:
    the same C ABI calls, so the same iterations bit for bit; the System-side parameter
    copy stepped by the stand-in optimiser stays on the engine's parameters."""
    if not os.path.exists(BIN):
        pytest.skip("integration/_build/b200_vmc is not built (needs the reference sources)")
    from vmachine_b200 import Engine
    text = DOT.format(steps=64 * 500, path=tmp_path) + "numWalkers: 64\n"
    cfg = tmp_path / "engine.in"
    cfg.write_text(text)
    r = subprocess.run([BIN, str(cfg), "engine", "3", "23"], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    lines = [json.loads(ln) for ln in r.stdout.splitlines() if ln.startswith("{")]
    assert len(lines) == 3
    with Engine(text) as e:
        e.init_walkers(None, seed=23)
        for it, ln in enumerate(lines):
            a = e.run_iteration(it)
            assert ln["energy"] == a.energy and ln["acceptance"] == a.acceptance
            assert ln["parameter_gap"] < 1e-14


@pytest.mark.gpu
def test_adapter_metropolis_matches_reference_program(tmp_path):
    """The reference's System::runSimulation, unchanged, with B200Metropolis moving its
    walker on the GPU from System's own random numbers, against the same program with
    its own ImportanceSampling: the same accept decisions, so the same iterations to the
    printed digits (the engine computes the moved coordinate in FP64 as the reference
    does, up to rounding)."""
    if not os.path.exists(BIN):
        pytest.skip("integration/_build/b200_vmc is not built (needs the reference sources)")
    out = {}
    for mode in ("reference", "metropolis"):
        d = tmp_path / mode
        d.mkdir()
        cfg = d / "input.in"
        cfg.write_text(DOT.format(steps=2000, path=d))
        r = subprocess.run([BIN, str(cfg), mode], capture_output=True, text=True, timeout=600)
        assert r.returncode == 0, r.stderr
        out[mode] = iteration_lines(r.stdout)
    (ref, ref_f), (gpu, gpu_f) = out["reference"], out["metropolis"]
    assert ref.shape == gpu.shape == (2, 10) and len(ref_f) == len(gpu_f) == 9
    assert np.allclose(gpu, ref, rtol=0, atol=2e-8), np.abs(gpu - ref).max()
    assert np.allclose(gpu_f, ref_f, rtol=0, atol=2e-10), np.abs(gpu_f - ref_f).max()
