"""The drop-in boundary without a GPU: the C-ABI library loads, exports every
entry point include/vmc_b200.h declares, and rejects bad input.in text the way
the reference's parser does (src/parser.cpp:314-320), before touching CUDA."""
import ctypes
import os
import re

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "vmc_b200.h")


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r"^\s*(?:int|void|long long|const char \*)\s*(vmc_\w+)\s*\(", text, re.M)))


def test_header_declares_entry_points():
    names = declared_functions()
    assert "vmc_create" in names and "vmc_sample" in names and "vmc_eval" in names
    assert len(names) >= 18


def test_library_exports_every_declared_symbol():
    from vmachine_b200 import EXPORTS, library
    lib = library()
    for name in declared_functions():
        assert hasattr(lib, name), name
    assert set(EXPORTS) <= set(declared_functions())
    version = int(re.search(r"#define VMC_ABI_VERSION (\d+)", open(HEADER).read()).group(1))
    assert lib.vmc_abi_version() == version


@pytest.mark.parametrize("text,code", [
    ("numParticles: 2\nbogusKey: 1\n", -1),
    ("numParticles: 2\nhamiltonian: harmonicOscillator\nwaveFunctionElement: gaussian\n"
     "sampling: metropolisHastings\n", -1),
    ("numParticles: 2\nhamiltonian: nothing\n", -1),
    ("numParticles: 2\nhamiltonian: harmonicOscillator\nwaveFunctionElement: fnn\n", -1),
    ("numParticles: 2\nhamiltonian: harmonicOscillator\nwaveFunctionElement: gaussian\n"
     "precision: fp16\n", -1),
    ("numParticles: 2\nhamiltonian: harmonicOscillator\nwaveFunctionElement: gaussian\n"
     "walkersPerWarp: 3\n", -1),
    # parsed, but not on the engine's path
    ("numParticles: 2\nhamiltonian: doubleWell 1.0\nwaveFunctionElement: gaussian\n", -2),
    ("numParticles: 4\nhamiltonian: harmonicOscillator\nwaveFunctionElement: slaterDeterminant\n"
     "basis: hermite\n", -2),
    ("numParticles: 2\nwaveFunctionElement: gaussian\n", -2),
    # hydrogen orbitals with n = 4 or l = 2 (hydrogenorbital.cpp:111-394: Ca, Z = 20, and
    # beyond) are not on the engine: only the closed shells up to Ar
    ("numParticles: 20\nnumDimensions: 3\natomicNumber: 20\nhamiltonian: atomicNucleus\n"
     "interactionStyle: coulomb\nwaveFunctionElement: slaterDeterminant\nbasis: hydrogenOrbital\n", -2),
    ("numParticles: 36\nnumDimensions: 3\natomicNumber: 36\nhamiltonian: atomicNucleus\n"
     "interactionStyle: coulomb\nwaveFunctionElement: slaterDeterminant\nbasis: hydrogenOrbital\n", -2),
    # the owner form of the production sweep covers the dots of N = 20 to 56
    ("numParticles: 12\nhamiltonian: harmonicOscillator\nwaveFunctionElement: slaterDeterminant\n"
     "waveFunctionElement: gaussian\nbasis: hermite\nsweepForm: owner\n", -2),
    ("numParticles: 12\nhamiltonian: harmonicOscillator\nwaveFunctionElement: gaussian\n"
     "sweepForm: fastest\n", -1),
    # the drift limiter: importance sampling in the corrected mode only
    ("numParticles: 2\nhamiltonian: harmonicOscillator\nwaveFunctionElement: gaussian\n"
     "sampling: importanceSampling\ndriftLimit: 0.5\n", -2),
    ("numParticles: 2\nhamiltonian: harmonicOscillator\nwaveFunctionElement: gaussian\n"
     "sampling: bruteForce\ncompat: corrected\ndriftLimit: 0.5\n", -2),
    ("numParticles: 2\nhamiltonian: harmonicOscillator\nwaveFunctionElement: gaussian\n"
     "compat: corrected\ndriftLimit: -1\n", -1),
])
def test_create_rejects(text, code):
    from vmachine_b200 import library
    lib = library()
    h = ctypes.c_void_p()
    rc = lib.vmc_create(text.encode(), None, ctypes.byref(h))
    assert rc == code, lib.vmc_last_error()
    assert not h.value
    assert lib.vmc_last_error()
