"""The MLP Jastrow oracle (oracle/mlp_jastrow.py) against finite differences:
gradient and Laplacian of J in the positions, dJ/dtheta in the parameters."""
import numpy as np
import pytest

from oracle import mlp_jastrow as mj


def random_theta(seed, scale=0.3):
    rng = np.random.default_rng(seed)
    return rng.normal(0.0, scale, mj.n_params())


@pytest.mark.parametrize("N,dim", [(2, 2), (6, 2), (8, 3)])
def test_position_derivatives(N, dim):
    theta = random_theta(N)
    x = np.random.default_rng(1).normal(0, 1.2, N * dim)
    J, G, lap = mj.jastrow(theta, x, N, dim)
    h = 1e-5
    Gn = np.zeros_like(G)
    Ln = 0.0
    for k in range(N * dim):
        e = np.zeros_like(x)
        e[k] = h
        jp, jm = mj.jastrow_value(theta, x + e, N, dim), mj.jastrow_value(theta, x - e, N, dim)
        Gn[k] = (jp - jm) / (2 * h)
        Ln += (jp - 2 * J + jm) / (h * h)
    assert np.max(np.abs(G - Gn)) < 1e-7 * max(1.0, np.max(np.abs(G)))
    assert abs(lap - Ln) < 1e-4 * max(1.0, abs(lap))


def test_parameter_gradient():
    N, dim = 6, 2
    theta = random_theta(3)
    x = np.random.default_rng(2).normal(0, 1.2, N * dim)
    g = mj.param_gradient(theta, x, N, dim, round_bf16=False)
    rng = np.random.default_rng(4)
    idx = np.concatenate([[0, 1, 130, 200, 4220, 4416, 4417, 4450, 5000, 5569], rng.integers(0, mj.n_params(), 30)])
    h = 1e-6
    for k in idx:
        e = np.zeros_like(theta)
        e[k] = h
        num = (mj.jastrow_value(theta + e, x, N, dim, False) -
               mj.jastrow_value(theta - e, x, N, dim, False)) / (2 * h)
        assert abs(g[k] - num) < 1e-6 * max(1.0, abs(num)), (k, g[k], num)


def test_bf16_rounding_and_layout():
    assert mj.n_params() == 5570
    # ties round to even: 1 + 2^-8 -> 1, 1 + 3 2^-8 -> 1 + 2^-6
    v = np.array([1.0, 1 + 2 ** -8, 1 + 3 * 2 ** -8, -3.14159265, 1e-3])
    r = mj.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0 and r[2] == 1 + 2 ** -6
    assert np.all(np.abs(r - v) <= np.abs(v) * 2 ** -8)
    t = mj.xavier(7)
    p = mj.unpack(t)
    assert np.all(p["w3"] == 0) and np.all(p["v3"] == 0)
    assert np.allclose(mj.pack(p), t)


@pytest.mark.parametrize("N,dim", [(6, 2), (8, 3)])
def test_symmetries(N, dim):
    """J depends on the pair distances, the pairs' spin and the radii only: exchanging
    two electrons of the same spin leaves J unchanged and exchanges their gradients;
    a rotation of all positions leaves J and the Laplacian unchanged and rotates the
    gradient.  Exchanging electrons of opposite spin changes J."""
    theta = random_theta(7)
    rng = np.random.default_rng(8)
    x = rng.normal(0, 1.2, (N, dim))
    J, G, lap = mj.jastrow(theta, x.ravel(), N, dim)
    G = G.reshape(N, dim)
    h = N // 2
    # same spin: particles 0 and 1 (both up), h and h + 1 (both down)
    for a, b in ((0, 1), (h, h + 1)):
        y = x.copy()
        y[[a, b]] = y[[b, a]]
        J2, G2, lap2 = mj.jastrow(theta, y.ravel(), N, dim)
        G2 = G2.reshape(N, dim)
        assert abs(J2 - J) < 1e-12 * max(1.0, abs(J))
        assert abs(lap2 - lap) < 1e-10 * max(1.0, abs(lap))
        assert np.allclose(G2[[b, a]], G[[a, b]], rtol=1e-12, atol=1e-12)
    y = x.copy()
    y[[0, h]] = y[[h, 0]]
    assert abs(mj.jastrow(theta, y.ravel(), N, dim)[0] - J) > 1e-6
    # a rotation about the origin
    q, _ = np.linalg.qr(rng.normal(size=(dim, dim)))
    Jr, Gr, lapr = mj.jastrow(theta, (x @ q.T).ravel(), N, dim)
    assert abs(Jr - J) < 1e-11 * max(1.0, abs(J))
    assert abs(lapr - lap) < 1e-9 * max(1.0, abs(lap))
    assert np.allclose(Gr.reshape(N, dim), G @ q.T, rtol=1e-10, atol=1e-10)
