"""Host-side restatement of the reference's per-iteration arithmetic (numpy, FP64).

TEST INFRASTRUCTURE ONLY: used by tests/ as the checker of the product's
iteration driver; never imported by the vmachine_b200 package.

- ``averages``: Sampler::computeAverages (src/sampler.cpp:194-226) over summed
  accumulators (the one-rank form of Sampler::computeTotals, :111-187).
- ``Adam``/``GradientDescent``: src/Optimization/adam.cpp:12-37 (m, v start at
  ones; beta1 0.89, beta2 0.999, eps 1e-8), gradientdescent.cpp / sgd.cpp:23-28
  (v starts at ones; v = gamma v + eta g / step^p), with
  g = 2(<E dlnPsi> - <E><dlnPsi>) (optimization.cpp:10-16) and theta -= update
  (system.cpp:114).
"""
import numpy as np

N_SCALARS = 9  # E, E^2, T, T^2, Vext, Vext^2, Vint, Vint^2, accepts


def averages(sums, n_samples, n_window, shape):
    """sums: accumulator vector summed over walkers; n_samples = total sampled steps;
    n_window = total gradient-window normaliser (walkers x steps-per-batch)."""
    s = np.asarray(sums, np.float64)
    M = float(n_samples)
    e, e2, t, t2, ve, ve2, vi, vi2, acc = s[:N_SCALARS] / np.array([M] * 8 + [1.0])
    ep = int(np.prod(shape))
    g = s[N_SCALARS:N_SCALARS + ep].reshape(shape) / n_window
    ge = s[N_SCALARS + ep:N_SCALARS + 2 * ep].reshape(shape) / n_window
    var = (e2 - e * e) / M
    return {
        "energy": e, "std_error": np.sqrt(var) if var > 0 else 0.0 * var, "kinetic": t,
        "external": ve, "interaction": vi, "acceptance": acc / M, "avg_grad": g, "avg_grad_e": ge,
    }


def energy_gradient(avg):
    return 2.0 * (avg["avg_grad_e"] - avg["energy"] * avg["avg_grad"])


class Adam:
    batches = 10

    def __init__(self, shape, eta):
        self.eta = eta
        self.m = np.ones(shape)
        self.v = np.ones(shape)
        self.t = 0

    def update(self, g):
        self.t += 1
        b1, b2, eps = 0.89, 0.999, 1e-8
        self.m = b1 * self.m + (1 - b1) * g
        self.v = b2 * self.v + (1 - b2) * g * g
        mh = self.m / (1 - b1 ** self.t)
        vh = self.v / (1 - b2 ** self.t)
        return self.eta * mh / (np.sqrt(vh) + eps)


class GradientDescent:
    batches = 1

    def __init__(self, shape, eta, gamma=0.0, power=0.0):
        self.eta, self.gamma, self.power = eta, gamma, power
        self.v = np.ones(shape)
        self.t = 0

    def update(self, g):
        self.t += 1
        self.v = self.gamma * self.v + self.eta * g * (1.0 / self.t ** self.power)
        return self.v
