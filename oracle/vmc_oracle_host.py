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
- ``Schedule``: System::runSimulation's iteration schedule (system.cpp:81-139) with
  adaptiveSteps (:213-224) and checkingConvergence (:197-208).
- ``DensityCounts``: the Sampler's radial, spatial and two-body densities
  (sampler.cpp:639-692), counted after every step as System::runMetropolisCycles
  does (system.cpp:147-164), with ``radial_vector_updated`` for which radial vector
  they see.
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


class Schedule:
    """System::runSimulation's schedule on one rank.

    The number of "normal" iterations is numIterations - rangeOfAdaptiveSteps - 1
    (system.cpp:92).  With adaptive steps, iteration `it` samples the initial step count
    times adaptiveSteps(): 2^additionalStepsLastIter at it == normal + range, the
    density iteration, 2^additionalSteps from `normal` on, else 1 (system.cpp:213-224).
    The convergence check keeps the last numberOfEnergies averages, shifted one place
    per iteration from zeros (userinput.cpp:196-202); when the first and the last
    differ by less than the tolerance, `normal` becomes it + 1 and the check stops
    (system.cpp:197-208).  The loop itself always runs numIterations times
    (system.cpp:93)."""

    def __init__(self, n_iterations, initial_steps, adaptive=False, range_=10, additional=4,
                 additional_last=5, check=False, n_energies=5, tolerance=1e-6):
        self.n_iterations, self.initial = n_iterations, initial_steps
        self.adaptive, self.range_ = adaptive, range_
        self.additional, self.additional_last = additional, additional_last
        self.check, self.tolerance = check, tolerance
        self.energies = np.zeros(n_energies)
        self.normal = n_iterations - range_ - 1

    def steps(self, it):
        if not self.adaptive:
            return self.initial
        if it == self.normal + self.range_:
            return self.initial * int(2 ** self.additional_last)
        if it >= self.normal:
            return self.initial * int(2 ** self.additional)
        return self.initial

    def is_density_iteration(self, it):
        return it == self.normal + self.range_

    def after(self, it, energy):
        if not self.check:
            return
        self.energies[:-1] = self.energies[1:].copy()
        self.energies[-1] = energy
        if abs(self.energies[0] - self.energies[-1]) < self.tolerance:
            self.normal = it + 1
            self.check = False


def radial_vector_updated(atomic_nucleus, hydrogenlike):
    """System::setGlobalArraysToCalculate (elementoperation.cpp:130-160): the
    Metropolis recomputes a moved particle's radius (importancesampling.cpp:64-66,
    bruteforce.cpp:38-40) only when an element, the Hamiltonian or the interaction
    asks for the radial vector.  Of the configured ones that is the atomic nucleus
    (atomicnucleus.h:16, need 3) and the hydrogen-like element (hydrogenlike.h:30,
    need 2); the Slater determinant, Gaussian, Pade, SimpleJastrow and RBM elements, the
    oscillator and Coulomb need none or the distance matrix only.  Otherwise System's
    radial vector keeps the initial state's radii."""
    return bool(atomic_nucleus or hydrogenlike)


class DensityCounts:
    """Sampler::computeOneBodyDensity (radial), computeOneBodyDensity2 (spatial, on the
    first two coordinates) and computeTwoBodyDensity (sampler.cpp:639-692) on `bins`
    bins of max_radius / bins, the spatial grid of twice that width centred on the
    origin (row = the y index), the two-body bins shifted by one (row = the
    lower-index particle).  C++ int() truncation toward zero is Python's int()."""

    def __init__(self, bins, max_radius):
        self.bins, self.half = bins, bins // 2
        self.max_radius, self.step = max_radius, max_radius / bins
        self.radial = np.zeros(bins, np.int64)
        self.spatial = np.zeros((bins, bins), np.int64)
        self.pair = np.zeros((bins, bins), np.int64)

    def add(self, positions, radii, d):
        n = len(radii)
        for r in radii:
            if r < self.max_radius:
                b = int(r / self.step)
                if b < self.bins:
                    self.radial[b] += 1
        x = np.asarray(positions, np.float64).reshape(n, d)
        for p in x:
            ix, iy = int(p[0] / (2 * self.step)), int(p[1] / (2 * self.step))
            if abs(ix) < self.half and abs(iy) < self.half:
                self.spatial[iy + self.half, ix + self.half] += 1
        for i in range(n):
            bi = int(radii[i] / self.step) + 1
            for j in range(i + 1, n):
                bj = int(radii[j] / self.step) + 1
                if bi < self.bins and bj < self.bins:
                    self.pair[bi, bj] += 1


def radii(positions, d):
    """Metropolis::calculateRadialVectorElement (metropolis.cpp:31-39): the square root
    of the particle's coordinates' squares, summed in order."""
    x = np.asarray(positions, np.float64).reshape(-1, d)
    out = np.zeros(len(x))
    for i, p in enumerate(x):
        acc = 0.0
        for v in p:
            acc += v * v
        out[i] = np.sqrt(acc)
    return out
