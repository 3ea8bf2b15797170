"""CPU oracle (test infrastructure only) for the learned MLP Jastrow factor.

The reference has no neural Jastrow on its `input.in` path, so this is a restatement
written from the mathematics, in FP64 numpy, checked by finite differences in the
tests.  Psi_J = exp(J) with

    J = sum_{i<j} u(r_ij, s_ij) + sum_i chi(r_i)

    u(r, s)  = a_s r / (1 + r) + w3 . tanh(W2 tanh(W1 [r, s] + b1) + b2) + b3
    chi(r)   = v3 . tanh(V2 tanh(V1 r + c1) + c2) + c3

s = 1 for a same-spin pair (both indices in the same half), else 0; a_s is the
cusp coefficient of the Pade-Jastrow (1/3 same spin, 1 opposite spin in 2D;
padejastrow.cpp:140-170).  The first term fixes the electron-electron cusp; the
network learns everything else.

Parameter vector (one row of the engine's E x p_max matrix), in this order:
W1 (H1 x 2, row-major [out][in]), b1 (H1), W2 (H2 x H1), b2 (H2), w3 (H2), b3,
V1 (G1), c1 (G1), V2 (G2 x G1), c2 (G2), v3 (G2), c3.
The engine evaluates the networks with the weights rounded to bfloat16 (round to
nearest even); `bf16` below gives the same rounding.
"""
import numpy as np

H1 = H2 = 64
G1 = G2 = 32


def n_params(h1=H1, h2=H2, g1=G1, g2=G2):
    return h1 * 2 + h1 + h2 * h1 + h2 + h2 + 1 + g1 + g1 + g2 * g1 + g2 + g2 + 1


def unpack(theta, h1=H1, h2=H2, g1=G1, g2=G2):
    t = np.asarray(theta, np.float64)
    out, o = {}, 0
    for name, shape in (("W1", (h1, 2)), ("b1", (h1,)), ("W2", (h2, h1)), ("b2", (h2,)),
                        ("w3", (h2,)), ("b3", ()), ("V1", (g1,)), ("c1", (g1,)),
                        ("V2", (g2, g1)), ("c2", (g2,)), ("v3", (g2,)), ("c3", ())):
        n = int(np.prod(shape)) if shape else 1
        out[name] = t[o:o + n].reshape(shape) if shape else t[o]
        o += n
    assert o == len(t), (o, len(t))
    return out


def bf16(x):
    """Round float64 values to bfloat16 (via float32, round to nearest even)."""
    f = np.asarray(x, np.float32).view(np.uint32).astype(np.uint64)
    r = ((f + 0x7FFF + ((f >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def xavier(seed, dim=2, h1=H1, h2=H2, g1=G1, g2=G2):
    """Xavier-uniform hidden layers from `seed`, zero output layers (J starts as the
    cusp term alone)."""
    rng = np.random.default_rng(seed)
    def xu(fo, fi, shape):
        lim = np.sqrt(6.0 / (fi + fo))
        return rng.uniform(-lim, lim, shape)
    p = dict(W1=xu(h1, 2, (h1, 2)), b1=np.zeros(h1), W2=xu(h2, h1, (h2, h1)), b2=np.zeros(h2),
             w3=np.zeros(h2), b3=0.0, V1=xu(g1, 1, (g1,)), c1=np.zeros(g1),
             V2=xu(g2, g1, (g2, g1)), c2=np.zeros(g2), v3=np.zeros(g2), c3=0.0)
    return pack(p)


def pack(p):
    return np.concatenate([np.ravel(p[k]) for k in
                           ("W1", "b1", "W2", "b2", "w3", "b3", "V1", "c1", "V2", "c2", "v3", "c3")])


def cusp_coef(dim, same):
    return np.where(same, 1.0 / 3 if dim == 2 else 1.0 / 4, 1.0 if dim == 2 else 0.5)


def pair_net(p, r, s, dim):
    """u, du/dr, d2u/dr2 for arrays r, s (forward-mode derivatives through tanh)."""
    r = np.asarray(r, np.float64)
    s = np.asarray(s, np.float64)
    a = cusp_coef(dim, s > 0.5)
    z1 = np.multiply.outer(r, p["W1"][:, 0]) + np.multiply.outer(s, p["W1"][:, 1]) + p["b1"]
    h1 = np.tanh(z1)
    g1 = 1.0 - h1 * h1
    d1 = g1 * p["W1"][:, 0]
    dd1 = -2.0 * h1 * g1 * p["W1"][:, 0] ** 2
    z2 = h1 @ p["W2"].T + p["b2"]
    dz2 = d1 @ p["W2"].T
    ddz2 = dd1 @ p["W2"].T
    h2 = np.tanh(z2)
    g2 = 1.0 - h2 * h2
    d2 = g2 * dz2
    dd2 = -2.0 * h2 * g2 * dz2 * dz2 + g2 * ddz2
    u = h2 @ p["w3"] + p["b3"] + a * r / (1.0 + r)
    du = d2 @ p["w3"] + a / (1.0 + r) ** 2
    ddu = dd2 @ p["w3"] - 2.0 * a / (1.0 + r) ** 3
    return u, du, ddu


def body_net(p, r):
    """chi, dchi/dr, d2chi/dr2."""
    r = np.asarray(r, np.float64)
    z1 = np.multiply.outer(r, p["V1"]) + p["c1"]
    h1 = np.tanh(z1)
    g1 = 1.0 - h1 * h1
    d1 = g1 * p["V1"]
    dd1 = -2.0 * h1 * g1 * p["V1"] ** 2
    z2 = h1 @ p["V2"].T + p["c2"]
    dz2 = d1 @ p["V2"].T
    ddz2 = dd1 @ p["V2"].T
    h2 = np.tanh(z2)
    g2 = 1.0 - h2 * h2
    return (h2 @ p["v3"] + p["c3"], (g2 * dz2) @ p["v3"],
            (-2.0 * h2 * g2 * dz2 * dz2 + g2 * ddz2) @ p["v3"])


def pairs(N):
    i, j = np.triu_indices(N, 1)
    h = N // 2
    same = ((i < h) == (j < h)).astype(np.float64)
    return i, j, same


def jastrow(theta, x, N, dim, round_bf16=True):
    """J, grad J (D), laplacian of J at positions x (D = N dim)."""
    p = unpack(bf16(theta) if round_bf16 else theta)
    X = np.asarray(x, np.float64).reshape(N, dim)
    i, j, same = pairs(N)
    dv = X[i] - X[j]
    r = np.sqrt((dv * dv).sum(1))
    u, du, ddu = pair_net(p, r, same, dim)
    ri = np.sqrt((X * X).sum(1))
    c, dc, ddc = body_net(p, ri)
    J = u.sum() + c.sum()
    G = np.zeros((N, dim))
    np.add.at(G, i, (du / r)[:, None] * dv)
    np.add.at(G, j, -(du / r)[:, None] * dv)
    G += (dc / ri)[:, None] * X
    lap = (2.0 * (ddu + (dim - 1) * du / r)).sum() + (ddc + (dim - 1) * dc / ri).sum()
    return J, G.ravel(), lap


def jastrow_value(theta, x, N, dim, round_bf16=True):
    return jastrow(theta, x, N, dim, round_bf16)[0]


def param_gradient(theta, x, N, dim, round_bf16=True):
    """dJ/dtheta (backpropagation through both networks, summed over pairs and
    particles) in the packed parameter order."""
    p = unpack(bf16(theta) if round_bf16 else theta)
    X = np.asarray(x, np.float64).reshape(N, dim)
    i, j, same = pairs(N)
    dv = X[i] - X[j]
    r = np.sqrt((dv * dv).sum(1))
    inp = np.stack([r, same], 1)
    h1 = np.tanh(inp @ p["W1"].T + p["b1"])
    h2 = np.tanh(h1 @ p["W2"].T + p["b2"])
    d2 = (1.0 - h2 * h2) * p["w3"]
    d1 = (d2 @ p["W2"]) * (1.0 - h1 * h1)
    g = dict(W1=d1.T @ inp, b1=d1.sum(0), W2=d2.T @ h1, b2=d2.sum(0), w3=h2.sum(0),
             b3=float(len(r)))
    ri = np.sqrt((X * X).sum(1))
    k1 = np.tanh(np.multiply.outer(ri, p["V1"]) + p["c1"])
    k2 = np.tanh(k1 @ p["V2"].T + p["c2"])
    e2 = (1.0 - k2 * k2) * p["v3"]
    e1 = (e2 @ p["V2"]) * (1.0 - k1 * k1)
    g.update(V1=e1.T @ ri, c1=e1.sum(0), V2=e2.T @ k1, c2=e2.sum(0), v3=k2.sum(0), c3=float(N))
    return pack(g)
