"""The engine's input.in parser against the reference's on the host.

The parsed settings (system size, omega and what it resets, Z and the hidden units and
what resets them, learning rate, steps, burn-in fraction, the driver's keys) equal the
reference System's after it parses the same text.  For every element set the engine
runs, the trial wave-function label (System::collectAllLabels,
parser.cpp:396-520: the element labels joined, then renamed by searchShortning,
:340-390), which Automatize reads to pick the initial weights
(InitialWeights/automatize.cpp), is the one the reference's own System builds from the
same text.  The parser (vmachine_b200/csrc/vmc_config.cpp) is compiled for the host
with tests/config_shim.cpp; the reference is the harness in oracle/_ref."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

from oracle_bind import (GAUSSIAN, HYDROGENLIKE, PADE, RBMGAUSSIAN, RBMPRODUCT, REF_SO, SIMPLEJASTROW,
                         SLATER, RefHarness, SystemSpec)

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
G, S, P, SJ, RG, RP, H = GAUSSIAN, SLATER, PADE, SIMPLEJASTROW, RBMGAUSSIAN, RBMPRODUCT, HYDROGENLIKE
ATOM = dict(d=3, atom=True, basis="hydrogenOrbital")

CASES = [
    ("gauss", SystemSpec(N=2, elements=(G,))),
    ("gauss_pade", SystemSpec(N=2, elements=(G, P))),
    ("pade_gauss", SystemSpec(N=2, elements=(P, G))),
    ("slater_gauss", SystemSpec(N=6, elements=(S, G))),
    ("gauss_slater", SystemSpec(N=6, elements=(G, S))),
    ("slater_gauss_pade", SystemSpec(N=6, elements=(S, G, P))),
    ("pade_slater_gauss", SystemSpec(N=6, elements=(P, S, G))),
    ("gauss_sj", SystemSpec(N=2, elements=(G, SJ))),
    ("slater_gauss_sj", SystemSpec(N=6, elements=(S, G, SJ))),
    ("rbm", SystemSpec(N=2, elements=(RG, RP), hidden=2)),
    ("rbm_reversed", SystemSpec(N=2, elements=(RP, RG), hidden=2)),
    ("rbm_pade", SystemSpec(N=2, elements=(RG, RP, P), hidden=2)),
    ("rbm_sj", SystemSpec(N=2, elements=(RG, RP, SJ), hidden=2)),
    ("he_slater_sj", SystemSpec(N=2, Z=2, elements=(S, SJ), **ATOM)),
    ("be_slater_pade", SystemSpec(N=4, Z=4, elements=(S, P), **ATOM)),
    ("he_slater", SystemSpec(N=2, Z=2, elements=(S,), **ATOM)),
    ("he_hydrogenlike", SystemSpec(N=2, d=3, Z=2, elements=(H,), atom=True)),
    ("he_hydrogenlike_pade", SystemSpec(N=2, d=3, Z=2, elements=(H, P), atom=True)),
]

NEEDS = pytest.mark.skipif(shutil.which("g++") is None or not os.path.exists(REF_SO),
                           reason="needs g++ and the reference harness")


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    """The engine's parser (vmc_config.cpp) and tests/config_shim.cpp built for the host."""
    out = str(tmp_path_factory.mktemp("cfgshim") / "libcfgshim.so")
    src = os.path.join(ROOT, "vmachine_b200", "csrc")
    subprocess.run(["g++", "-std=c++17", "-O1", "-shared", "-fPIC", "-I", src,
                    os.path.join(HERE, "config_shim.cpp"), os.path.join(src, "vmc_config.cpp"),
                    "-o", out], check=True)
    lib = ctypes.CDLL(out)
    lib.cfg_trial_label.restype = ctypes.c_long
    lib.cfg_trial_label.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_long]
    lib.cfg_settings.restype = ctypes.c_int
    lib.cfg_settings.argtypes = [ctypes.c_char_p, ctypes.c_void_p]
    lib.cfg_parameter_counts.restype = ctypes.c_int
    lib.cfg_parameter_counts.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int]
    return lib


@NEEDS
@pytest.mark.parametrize("name,spec", CASES, ids=[c[0] for c in CASES])
def test_trial_label_matches_reference(shim, name, spec):
    text = spec.input_in()
    buf = ctypes.create_string_buffer(512)
    n = shim.cfg_trial_label(text.encode(), buf, len(buf))
    assert n >= 0, f"the engine's parser rejected {name}"
    ours = buf.raw[:n].decode()
    ref = RefHarness(spec, np.random.default_rng(1).normal(0.0, 1.0, spec.D))
    try:
        theirs = ref.trial_label()
    finally:
        ref.close()
    assert ours == theirs, (name, ours, theirs)


@NEEDS
@pytest.mark.parametrize("name,spec", CASES, ids=[c[0] for c in CASES])
def test_parameter_counts_match_reference(shim, name, spec):
    """The parameter matrix has the reference's shape: as many rows as elements and
    as many columns as the largest element's parameter count (System::setMaxParameters,
    elementoperation.cpp:173-186), with each element's count from the engine's
    element_parameters."""
    lib = shim
    counts = np.zeros(16, np.int32)
    n = lib.cfg_parameter_counts(spec.input_in().encode(), counts.ctypes.data, len(counts))
    assert n == len(spec.elements)
    ref = RefHarness(spec, np.random.default_rng(1).normal(0.0, 1.0, spec.D))
    try:
        E, P = ref.E, ref.P
    finally:
        ref.close()
    assert (n, int(counts[:n].max())) == (E, P), (name, counts[:n], E, P)


SETTINGS = ("particles", "dimensions", "omega", "sigma", "Z", "hidden units", "learning rate",
            "iterations", "equilibration fraction", "total steps", "step length", "sorting",
            "max radius", "bins", "tolerance", "energies", "range of adaptive steps",
            "additional steps", "additional steps last", "checkpoint frequency", "check convergence",
            "adaptive steps", "one-body density", "spatial density", "two-body density")

BODY = ["hamiltonian: harmonicOscillator", "interactionStyle: coulomb", "waveFunctionElement: gaussian",
        "waveFunctionElement: padeJastrow", "sampling: importanceSampling", "optimization: adam",
        "numSteps: 1000", "numIterations: 12"]

SETTING_CASES = [
    # main.cpp's defaults and system.h's
    ("defaults", ["numParticles: 2", "numDimensions: 2"]),
    # omega: resets stepLength to 0.1 / sqrt(omega) and the RBM width (parser.cpp:57-60)
    ("omega_then_step", ["numParticles: 2", "omega: 0.5", "stepLength: 0.2"]),
    ("step_then_omega", ["numParticles: 2", "stepLength: 0.2", "omega: 0.5"]),
    # numParticles: resets Z and the hidden units (parser.cpp:51-54)
    ("hidden_then_particles", ["numHiddenNodes: 3", "numParticles: 6"]),
    ("particles_then_hidden", ["numParticles: 6", "numHiddenNodes: 3"]),
    ("z_then_particles", ["atomicNumber: 3", "numParticles: 4"]),
    ("particles_then_z", ["numParticles: 4", "atomicNumber: 3"]),
    # the driver's keys
    ("driver", ["numParticles: 2", "learningRate: 0.02", "equilibration: 0.01", "sorting: false",
                "maxRadius: 3.0", "numberOfBins: 50", "checkConvergence: true", "numberOfEnergies: 7",
                "tolerance: 1e-5", "applyAdaptiveSteps: true", "rangeOfAdaptiveSteps: 4",
                "additionalSteps: 2", "additionalStepsLastIter: 3", "checkpointFreq: 10",
                "computeOneBodyDensity: true", "computeOneBodyDensity2: true",
                "computeTwoBodyDensity: true"]),
]


@NEEDS
@pytest.mark.parametrize("name,lines", SETTING_CASES, ids=[c[0] for c in SETTING_CASES])
def test_parsed_settings_match_reference(shim, name, lines):
    """The same input.in text through the engine's parser and the reference's
    (System::parser and its set-up) gives the same settings, key side effects included."""
    text = "\n".join(lines + BODY) + "\n"
    lib = shim
    ours = np.zeros(len(SETTINGS))
    assert lib.cfg_settings(text.encode(), ours.ctypes.data) == len(SETTINGS)
    N = int(ours[0])
    ref = RefHarness(None, np.random.default_rng(1).normal(0.0, 1.0, 2 * N), text=text)
    try:
        theirs = ref.settings()
    finally:
        ref.close()
    assert len(theirs) == len(SETTINGS)
    diff = [(k, a, b) for k, a, b in zip(SETTINGS, ours, theirs) if not np.isclose(a, b, rtol=1e-15, atol=0)]
    assert not diff, (name, diff)
