"""Checkpoint and resume on the GPU: an engine resumed from a walker-state file
continues exactly as the engine that saved it; parameter files round-trip through
vmc_write_weights / vmc_read_weights; vmc_run_simulation writes weights_<it>.dat
every checkpointFreq iterations like the reference (system.cpp:116-118)."""
import os

import numpy as np
import pytest

from vmachine_b200.batch import atom_text, dot_text
from vmachine_b200.learned import dot_config

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("text", [dot_text(6, 0.6, 96, 400, "mixed", seed=3),
                                  dot_text(12, 0.8, 64, 300, "fp64", seed=4),
                                  dot_text(56, 0.28, 40, 300, "mixed", seed=6),
                                  atom_text(2, 32, 300, seed=5),
                                  dot_config(6, 1.0, "mlpJastrow", 64, 200, 3e-4)],
                         ids=["dot6-mixed", "dot12-fp64", "dot56-mixed-owner", "he-general", "mlp-dot-mixed"])
def test_exact_restart(tmp_path, text):
    from vmachine_b200 import Engine
    path = tmp_path / "state.bin"
    with Engine(text) as a:
        a.init_walkers(None, seed=11)
        for it in range(3):
            a.run_iteration(it)
        a.save_state(path)
        ea = [a.run_iteration(it).energy for it in range(3, 6)]
        pa, xa, ra = a.parameters(), a.positions(), a.refresh_interval()
    with Engine(text) as b:
        b.load_state(path)
        eb = [b.run_iteration(it).energy for it in range(3, 6)]
        pb, xb, rb = b.parameters(), b.positions(), b.refresh_interval()
    assert ea == eb
    assert np.array_equal(xa, xb) and ra == rb
    if "mlpJastrow" in text:
        # the MLP row's gradient sums are FP64 atomics of the backward kernel, whose
        # order varies from run to run: the parameters agree to rounding (the sampled
        # energies above, which see the bfloat16-rounded weights, are identical)
        assert np.allclose(pa, pb, rtol=1e-12, atol=1e-15)
    else:
        assert np.array_equal(pa, pb)


def test_state_file_for_another_system_is_rejected(tmp_path):
    from vmachine_b200 import Engine, VmcError
    path = tmp_path / "state.bin"
    with Engine(dot_text(6, 0.6, 96, 400, seed=3)) as a:
        a.init_walkers(None, seed=1)
        a.save_state(path)
    with Engine(dot_text(6, 0.6, 64, 400, seed=3)) as b:
        with pytest.raises(VmcError, match="walkers"):
            b.load_state(path)


def test_weights_round_trip(tmp_path):
    from vmachine_b200 import Engine
    text = dot_text(6, 0.6, 32, 200, seed=3)
    with Engine(text) as a:
        a.init_walkers(None, seed=1)
        a.run_iteration(0)
        a.write_weights(tmp_path / "w.dat", 17)
        a.write_weights(tmp_path / "w6.dat")
        th = a.parameters()
    with Engine(text) as b:
        b.init_walkers(None, seed=1)
        b.read_weights(tmp_path / "w.dat")
        assert np.array_equal(b.parameters(), th)
    six = np.loadtxt(tmp_path / "w6.dat", ndmin=2)
    assert np.allclose(six, th, rtol=1e-5, atol=1e-6)


def test_run_simulation_checkpoints(tmp_path):
    from vmachine_b200 import Engine
    text = dot_text(6, 0.6, 32, 200, seed=3) + "\n".join(
        ["numIterations: 5", "printParametersToFile: true", "checkpointFreq: 2", f"path: {tmp_path}/"]) + "\n"
    with Engine(text) as e:
        e.init_walkers(None, seed=2)
        e.run_simulation()
        th = e.parameters()
    assert sorted(f for f in os.listdir(tmp_path) if f.startswith("weights_")) == \
        ["weights_0.dat", "weights_2.dat", "weights_4.dat"]
    last = np.loadtxt(tmp_path / "weights_4.dat", ndmin=2)
    assert np.allclose(last, th, rtol=1e-5, atol=1e-6)


def _state_sections(raw):
    """(offset, size) of each section of a walker-state file: the header is "VMCSTATE",
    u32 version, u32 n, n i32 header values, u64 seed, f64 previous gamma; each section
    is a u64 byte count and the bytes (theta, opt_m, opt_v, records, scalars, masks,
    counters, status words, MLP caches)."""
    import struct
    nh = struct.unpack_from("<I", raw, 12)[0]
    off = 16 + 4 * nh + 16
    out = []
    while off < len(raw):
        n = struct.unpack_from("<Q", raw, off)[0]
        out.append((off + 8, n))
        off += 8 + n
    return out


def test_timed_out_walkers_fail_the_pass(tmp_path):
    """A walker whose status word carries the tensor-core timeout bit (a CTA that gave
    up waiting stops sampling part-way) makes vmc_sample fail with VMC_E_TIMEOUT instead
    of returning biased sums, and the parameters stay put; vmc_init_walkers clears it.
    The bit is set in a saved walker-state file (no device wait is made to expire)."""
    import struct
    from vmachine_b200 import Engine, VmcError
    text = dot_text(6, 0.6, 64, 200, "mixed", seed=3)
    path = tmp_path / "state.bin"
    with Engine(text) as a:
        a.init_walkers(None, seed=1)
        a.run_iteration(0)
        a.save_state(path)
    raw = bytearray(path.read_bytes())
    off, n = _state_sections(raw)[7]  # the status words
    assert n == 64 * 4
    struct.pack_into("<I", raw, off + 4 * 5, 8)  # walker 5: ST_TC_TIMEOUT
    path.write_bytes(bytes(raw))
    with Engine(text) as b:
        b.load_state(path)
        th = b.parameters()
        with pytest.raises(VmcError) as err:
            b.run_iteration(1)
        assert err.value.code == -8
        assert np.array_equal(b.parameters(), th)
        b.init_walkers(None, seed=2)
        assert np.isfinite(b.run_iteration(1).energy)
