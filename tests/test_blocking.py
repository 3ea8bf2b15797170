"""The engine's Blocker (vmc_block_series, the host form of the device blocking
test) against the reference's Blocker outputs (tests/golden/blocking.npz) and the C
oracle (oracle/vmc_oracle.c vmo_blocking) on correlated series."""
import os

import numpy as np
import pytest

from oracle_bind import Oracle, load_cases

HERE = os.path.dirname(os.path.abspath(__file__))
BLOCK = load_cases(os.path.join(HERE, "golden", "blocking.npz"))


def ar1(n, phi, seed):
    rng = np.random.default_rng(seed)
    e = rng.normal(size=n)
    x = np.empty(n)
    x[0] = e[0]
    for i in range(1, n):
        x[i] = phi * x[i - 1] + e[i]
    return 3.0 + 0.1 * x


@pytest.mark.parametrize("name", sorted(BLOCK))
def test_golden(name):
    from vmachine_b200 import block_series
    c = BLOCK[name]
    b = block_series(c["x"])
    assert abs(b.mean - float(c["mean"])) < 1e-12 * max(1.0, abs(float(c["mean"])))
    assert abs(b.std_error - float(c["std_error"])) < 1e-9 * float(c["std_error"])


@pytest.mark.parametrize("n,phi,seed", [(2, 0.0, 1), (64, 0.5, 2), (1024, 0.9, 3), (1 << 14, 0.99, 4),
                                        (1 << 16, 0.3, 5), (1 << 12, -0.6, 6)])
def test_against_oracle(n, phi, seed):
    from vmachine_b200 import block_series
    x = ar1(n, phi, seed)
    mean, var = Oracle().blocking(x)
    b = block_series(x)
    assert abs(b.mean - mean) < 1e-13 * abs(mean)
    assert abs(b.mse_mean - var) <= 1e-12 * var
    nk = b.n_k
    assert nk >= 2 and (nk & (nk - 1)) == 0
    assert abs(b.mse_std_error - (2 * nk - 1) * var * var / nk ** 2) <= 1e-12 * b.mse_std_error


def test_not_power_of_two_and_constant():
    from vmachine_b200 import block_series
    b = block_series(np.ones(1000))
    assert b.mean == -1.0 and b.std_error == -1.0 and b.n_k == 0
    c = block_series(np.full(256, 2.0))
    assert c.mean == 2.0 and c.std_error == 0.0


def test_reference_resampling_example():
    """The reference's own Blocker fixture: examples/resampling/523861_0.dat, the
    instant energies (2^17) of that example's last iteration, whose blocked result the
    example's log prints as 'Total energy : 3.0111013667 (with STD = 0.0030690608)';
    also against the reference's Blocker compiled from its sources (oracle/_ref)."""
    import ctypes
    from vmachine_b200 import block_series
    ref = os.environ.get("VMC_REFERENCE_DIR", "/root/reference")
    path = os.path.join(ref, "examples", "resampling", "523861_0.dat")
    if not os.path.exists(path):
        pytest.skip("the reference's example files are not on this machine")
    x = np.loadtxt(path)
    assert len(x) == 1 << 17
    b = block_series(x)
    assert round(b.mean, 10) == 3.0111013667 and round(b.std_error, 10) == 0.0030690608
    so = os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libvmref.so")
    if os.path.exists(so):
        lib = ctypes.CDLL(so)
        lib.vmref_blocking.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p]
        out = np.zeros(2)
        lib.vmref_blocking(x.ctypes.data_as(ctypes.c_void_p), len(x), out.ctypes.data_as(ctypes.c_void_p))
        assert abs(b.mean - out[0]) < 1e-14 * abs(out[0]) and abs(b.std_error - out[1]) < 1e-12 * out[1]
