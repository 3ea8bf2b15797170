"""vmc_local_energies_noalloc (include/vmc_b200.h) through the C ABI, against the
engine's own FP64 evaluation at the same positions (vmc_init_walkers with host
positions, then vmc_eval).

Both paths run the same FP64 rebuild and evaluation kernels on the same inputs,
so the energies agree to rounding; the bar here is 1e-12 relative (max-abs over
the array relative to its max-abs).  Two calls in a row with different positions
check that nothing left in the shared scratch array by the first call reaches
the second.  The test allocates the position and energy buffers itself (torch);
the entry point allocates nothing.
"""
import ctypes

import numpy as np
import pytest

from oracle_bind import GAUSSIAN, HYDROGENLIKE, PADE, SLATER, SystemSpec

pytestmark = pytest.mark.gpu

TOL = 1e-12

CASES = {
    # closed-shell quantum dot, Coulomb, importance sampling, reference quirks on
    "dot6": (SystemSpec(N=6, d=2, elements=[GAUSSIAN, SLATER, PADE], omega=1.0, coulomb=True,
                        sampling="importanceSampling"), [0.93, 0.0, 0.41], 64),
    # the headline system: 56 electrons at omega = 0.28
    "dot56": (SystemSpec(N=56, d=2, elements=[GAUSSIAN, SLATER, PADE], omega=0.28, coulomb=True,
                         sampling="importanceSampling"), [1.02, 0.0, 0.36], 200),
    # helium-like atom in 3D, brute-force sampling
    "atom3d": (SystemSpec(N=2, d=3, elements=[HYDROGENLIKE, PADE], atom=True, Z=2, coulomb=True,
                          sampling="bruteForce"), [0.88, 0.5], 96),
}


def entry():
    from vmachine_b200 import library
    lib = library()
    f = lib.vmc_local_energies_noalloc
    f.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
                  ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
    f.restype = ctypes.c_int
    return lib, f


def rel(a, b):
    scale = max(float(np.max(np.abs(b))), 1e-300)
    return float(np.max(np.abs(a - b)) / scale)


def positions(rng, W, D, scale):
    return rng.normal(0.0, scale, size=(W, D))


@pytest.mark.parametrize("name", sorted(CASES))
def test_two_calls_match_engine_eval(name):
    import torch
    from vmachine_b200 import Engine
    spec, theta, W = CASES[name]
    text = spec.input_in()
    theta = np.asarray(theta, np.float64).reshape(len(theta), 1)
    D = spec.N * spec.d
    rng = np.random.default_rng(17)
    scale = 1.0 / np.sqrt(spec.omega) if not spec.atom else 0.8
    lib, f = entry()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    energies = torch.full((W, 3), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    with Engine(text, walkers=W, precision=0) as eng:
        eng.set_parameters(theta)
        for call in range(2):
            pos = positions(rng, W, D, scale * (1.0 + 0.25 * call))
            eng.init_walkers(pos)
            _, _, _, want = eng.eval()
            d_pos = torch.from_numpy(pos).to(dev)
            torch.cuda.synchronize(dev)
            rc = f(text.encode(), theta.ctypes.data, theta.shape[0], theta.shape[1],
                   d_pos.data_ptr(), W, energies.data_ptr(), stream.cuda_stream)
            assert rc == 0, lib.vmc_last_error()
            stream.synchronize()
            got = energies.cpu().numpy()
            assert np.all(np.isfinite(got))
            assert rel(got, want) < TOL, (call, rel(got, want))


def test_matches_reference_fixture_n56():
    """The headline system's energies at the reference-generated fixed positions
    (tests/golden/eval_fixed.npz, the reference's own evaluation): kinetic, external
    and interaction energy of three walkers, 1e-10 relative."""
    import os

    import torch
    from oracle_bind import load_cases, spec_from_case
    c = load_cases(os.path.join(os.path.dirname(__file__), "golden", "eval_fixed.npz"))["n56_w028_slater_gauss_pade"]
    spec = spec_from_case(c)
    pos = np.ascontiguousarray(c["pos"], np.float64)
    theta = np.ascontiguousarray(c["theta"], np.float64)
    W = pos.shape[0]
    lib, f = entry()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    d_pos = torch.from_numpy(pos).to(dev)
    energies = torch.full((W, 3), float("nan"), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    rc = f(spec.input_in().encode(), theta.ctypes.data, theta.shape[0], theta.shape[1], d_pos.data_ptr(), W,
           energies.data_ptr(), stream.cuda_stream)
    assert rc == 0, lib.vmc_last_error()
    stream.synchronize()
    assert rel(energies.cpu().numpy(), c["energies"]) < 1e-10


def test_call_leaves_device_memory_unchanged():
    """After the first call on the device (its one-time set-up), a call changes the
    device's free memory by nothing: the entry point allocates no device memory."""
    import torch
    spec, theta, W = CASES["dot56"]
    theta = np.asarray(theta, np.float64).reshape(len(theta), 1)
    lib, f = entry()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    rng = np.random.default_rng(5)
    d_pos = torch.from_numpy(positions(rng, W, spec.N * spec.d, 1.0 / np.sqrt(spec.omega))).to(dev)
    energies = torch.zeros((W, 3), dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)
    args = (spec.input_in().encode(), theta.ctypes.data, theta.shape[0], theta.shape[1], d_pos.data_ptr(), W,
            energies.data_ptr(), stream.cuda_stream)
    assert f(*args) == 0, lib.vmc_last_error()  # first call: the per-device set-up
    stream.synchronize()
    free_before, _ = torch.cuda.mem_get_info(dev)
    for _ in range(3):
        assert f(*args) == 0, lib.vmc_last_error()
    stream.synchronize()
    free_after, _ = torch.cuda.mem_get_info(dev)
    assert free_after == free_before
    assert np.all(np.isfinite(energies.cpu().numpy()))


def test_rejects_walker_counts_beyond_the_array():
    import torch
    spec, theta, _ = CASES["dot56"]
    theta = np.asarray(theta, np.float64).reshape(len(theta), 1)
    lib, f = entry()
    dev = torch.device("cuda", 0)
    buf = torch.zeros(8, dtype=torch.float64, device=dev)
    rc = f(spec.input_in().encode(), theta.ctypes.data, 3, 1, buf.data_ptr(), 100000,
           buf.data_ptr(), None)
    assert rc == -4
    msg = lib.vmc_last_error().decode()
    assert "bytes of scratch" in msg and "at most" in msg
    # the shape check comes before any device work too
    rc = f(spec.input_in().encode(), theta.ctypes.data, 2, 1, buf.data_ptr(), 4, buf.data_ptr(), None)
    assert rc == -4 and b"shape" in lib.vmc_last_error()
