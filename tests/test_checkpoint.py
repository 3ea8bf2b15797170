"""Parameter files in the reference's format without a GPU: the engine's writer
against the reference's own output (tests/golden/weights_format.npz, written by
Sampler::printParametersToFile's Eigen stream format), and the reference's FromFile
reading the engine's full-precision files back (when the reference harness is
built)."""
import ctypes
import os

import numpy as np
import pytest

from oracle_bind import GAUSSIAN, PADE, REF_SO, SLATER, RefHarness, SystemSpec, load_cases

HERE = os.path.dirname(os.path.abspath(__file__))
CASES = load_cases(os.path.join(HERE, "golden", "weights_format.npz"))


def fmt(theta, digits=0):
    from vmachine_b200 import library
    lib = library()
    lib.vmc_format_weights.restype = ctypes.c_longlong
    lib.vmc_format_weights.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_char_p,
                                       ctypes.c_longlong]
    th = np.ascontiguousarray(theta, np.float64)
    buf = ctypes.create_string_buffer(1 << 16)
    n = lib.vmc_format_weights(th.ctypes.data_as(ctypes.c_void_p), th.shape[0], th.shape[1], digits, buf, len(buf))
    assert 0 < n < len(buf)
    return buf.value.decode()


@pytest.mark.parametrize("name", sorted(CASES))
def test_reference_text(name):
    c = CASES[name]
    assert fmt(c["theta"]) == str(c["text"])


def test_full_precision_round_trip(tmp_path):
    rng = np.random.default_rng(3)
    th = rng.normal(size=(3, 7)) * 10.0 ** rng.integers(-8, 8, size=(3, 7))
    text = fmt(th, 17)
    back = np.array([[float(v) for v in line.split()] for line in text.splitlines() if line.strip()])
    assert np.array_equal(back, th)


@pytest.mark.skipif(not os.path.exists(REF_SO), reason="reference harness not built (make -C oracle ref)")
def test_reference_reads_engine_file(tmp_path):
    th = np.array([[0.0], [0.812345678901234], [0.3398765432101234]])
    path = tmp_path / "weights_7.dat"
    path.write_text(fmt(th, 17))
    spec = SystemSpec(N=6, elements=(SLATER, GAUSSIAN, PADE), extra=[f"initialWeights: fromfile {path}"])
    h = RefHarness(spec, np.zeros(12))
    got = np.zeros(3)
    h.lib.vmref_get_params(h.h, got.ctypes.data_as(ctypes.c_void_p))
    h.close()
    assert np.array_equal(got, th.ravel())
