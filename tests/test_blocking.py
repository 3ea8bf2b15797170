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
