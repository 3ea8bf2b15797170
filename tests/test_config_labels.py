"""The engine's input.in parser against the reference's on the host: for every
element set the engine runs, the trial wave-function label (System::collectAllLabels,
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

SHIM = None


def shim():
    global SHIM
    if SHIM is None:
        import tempfile
        out = os.path.join(tempfile.mkdtemp(prefix="cfgshim_"), "libcfgshim.so")
        src = os.path.join(ROOT, "vmachine_b200", "csrc")
        subprocess.run(["g++", "-std=c++17", "-O1", "-shared", "-fPIC", "-I", src,
                        os.path.join(HERE, "config_shim.cpp"), os.path.join(src, "vmc_config.cpp"),
                        "-o", out], check=True)
        SHIM = ctypes.CDLL(out)
        SHIM.cfg_trial_label.restype = ctypes.c_long
        SHIM.cfg_trial_label.argtypes = [ctypes.c_char_p, ctypes.c_char_p, ctypes.c_long]
    return SHIM


@pytest.mark.skipif(shutil.which("g++") is None or not os.path.exists(REF_SO),
                    reason="needs g++ and the reference harness")
@pytest.mark.parametrize("name,spec", CASES, ids=[c[0] for c in CASES])
def test_trial_label_matches_reference(name, spec):
    text = spec.input_in()
    buf = ctypes.create_string_buffer(512)
    n = shim().cfg_trial_label(text.encode(), buf, len(buf))
    assert n >= 0, f"the engine's parser rejected {name}"
    ours = buf.raw[:n].decode()
    ref = RefHarness(spec, np.random.default_rng(1).normal(0.0, 1.0, spec.D))
    try:
        theirs = ref.trial_label()
    finally:
        ref.close()
    assert ours == theirs, (name, ours, theirs)
