"""ctypes bindings for the two CPU checkers (test infrastructure only).

- ``Oracle``: the C restatement in oracle/vmc_oracle.c (liboracle.so).
- ``RefHarness``: the reference's own C++ classes built from its sources by
  oracle/Makefile (oracle/_ref/libvmref.so); present only where the reference
  sources could be compiled (this container), never on the GPU box.

``SystemSpec`` describes one system both ways: as input.in text (the reference
parses it) and as the oracle's ``vmo_system`` struct.
"""
import ctypes
import os
from dataclasses import dataclass, field

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "liboracle.so")
REF_SO = os.path.join(ROOT, "oracle", "_ref", "libvmref.so")

GAUSSIAN, SLATER, PADE, SIMPLEJASTROW, RBMGAUSSIAN, RBMPRODUCT, HYDROGENLIKE = range(7)
ELEMENT_KEYS = {
    GAUSSIAN: "gaussian", SLATER: "slaterDeterminant", PADE: "padeJastrow",
    SIMPLEJASTROW: "simpleJastrow", RBMGAUSSIAN: "RBMGaussian", RBMPRODUCT: "RBMProduct",
    HYDROGENLIKE: "hydrogenLike",
}
Q_PADE_RATIO, Q_PADE_DGAMMA, Q_SJ_RATIO, Q_IS_GREEN, Q_RBM_SORT, Q_HORB3 = 1, 2, 4, 8, 16, 32
Q_ALL = 63

_dp = ctypes.POINTER(ctypes.c_double)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p) if a is not None else None


class VmoSystem(ctypes.Structure):
    _fields_ = [
        ("N", ctypes.c_int), ("d", ctypes.c_int), ("n_elem", ctypes.c_int),
        ("elem", ctypes.c_int * 8), ("basis", ctypes.c_int), ("hamiltonian", ctypes.c_int),
        ("coulomb", ctypes.c_int), ("sampling", ctypes.c_int), ("hidden", ctypes.c_int),
        ("p_max", ctypes.c_int), ("quirks", ctypes.c_int), ("omega", ctypes.c_double),
        ("Z", ctypes.c_double), ("step", ctypes.c_double), ("sigma", ctypes.c_double),
        ("drift_limit", ctypes.c_double),
    ]


@dataclass
class SystemSpec:
    N: int = 2
    d: int = 2
    elements: tuple = (GAUSSIAN, PADE)
    omega: float = 1.0
    Z: int = 0
    coulomb: bool = True
    sampling: str = "importanceSampling"   # or "bruteForce"
    step: float = 0.1                      # stepLength (dt for importance sampling)
    hidden: int = 2
    atom: bool = False                     # atomicNucleus Hamiltonian instead of harmonic oscillator
    basis: str = "hermite"
    sorting: bool = False
    drift_limit: float = 0.0               # corrected importance sampling: drift limiter a (0: off)
    optimization: str = "adam"
    learning_rate: float = 0.1
    num_steps: int = 1000
    quirks: int = Q_ALL
    extra: list = field(default_factory=list)

    @property
    def D(self):
        return self.N * self.d

    def n_params(self, e):
        el = self.elements[e]
        if el == SLATER:
            return 0
        if el == SIMPLEJASTROW:
            return self.N * self.N
        if el == RBMGAUSSIAN:
            return self.D
        if el == RBMPRODUCT:
            return self.hidden * self.D + self.hidden
        return 1

    @property
    def p_max(self):
        return max(self.n_params(e) for e in range(len(self.elements)))

    def input_in(self):
        """input.in text in the reference's key schema (parser.cpp:51-313)."""
        L = [f"numParticles: {self.N}", f"numDimensions: {self.d}"]
        if self.atom:
            L += [f"atomicNumber: {self.Z}", "hamiltonian: atomicNucleus"]
        else:
            L += ["hamiltonian: harmonicOscillator", f"omega: {self.omega!r}"]
        if self.coulomb:
            L.append("interactionStyle: coulomb")
        for e in self.elements:
            L.append(f"waveFunctionElement: {ELEMENT_KEYS[e]}")
        if SLATER in self.elements:
            L.append(f"basis: {self.basis}")
        if RBMPRODUCT in self.elements:
            L.append(f"numHiddenNodes: {self.hidden}")
        L.append(f"sorting: {'true' if self.sorting else 'false'}")
        L.append(f"sampling: {self.sampling}")
        L.append(f"stepLength: {self.step!r}")
        if self.drift_limit > 0:
            L.append(f"driftLimit: {self.drift_limit!r}")
        L.append(f"optimization: {self.optimization}")
        L.append(f"learningRate: {self.learning_rate!r}")
        L.append(f"numSteps: {self.num_steps}")
        L += self.extra
        return "\n".join(L) + "\n"

    def vmo(self):
        s = VmoSystem()
        s.N, s.d, s.n_elem = self.N, self.d, len(self.elements)
        for i, e in enumerate(self.elements):
            s.elem[i] = e
        s.basis = 1 if self.basis == "hermite" else 2
        s.hamiltonian = 1 if self.atom else 0
        s.coulomb = int(self.coulomb)
        s.sampling = 0 if self.sampling == "importanceSampling" else 1
        s.hidden = self.hidden
        s.p_max = self.p_max
        quirks = self.quirks
        if not self.sorting:
            quirks &= ~Q_RBM_SORT
        s.quirks = quirks
        s.omega = self.omega
        s.Z = float(self.Z)
        s.step = self.step
        s.sigma = 1.0 / np.sqrt(self.omega) if not self.atom else 1.0
        s.drift_limit = self.drift_limit
        return s


class Oracle:
    def __init__(self, path=ORACLE_SO):
        self.lib = ctypes.CDLL(path)
        for name in ("vmo_eval", "vmo_ratio", "vmo_run", "vmo_quantum_force"):
            getattr(self.lib, name).restype = ctypes.c_int
        self.lib.vmo_blocking.restype = ctypes.c_double
        self.lib.vmo_ratio.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_int, ctypes.c_double, ctypes.c_void_p]
        self.lib.vmo_step_randoms.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_uint64,
                                              ctypes.c_int, ctypes.c_void_p]
        self.lib.vmo_initial_positions.argtypes = [ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int,
                                                   ctypes.c_int, ctypes.c_double, ctypes.c_void_p]
        self.lib.vmo_blocking.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p]
        self.lib.vmo_run.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_int, ctypes.c_int,
                                     ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_uint64,
                                     ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
                                     ctypes.c_void_p]

    def eval(self, spec, theta, pos):
        s = spec.vmo()
        E, D, P = len(spec.elements), spec.D, spec.p_max
        grad, lap = np.zeros(E * D), np.zeros(E)
        pgrad, en = np.zeros(E * P), np.zeros(3)
        theta = np.ascontiguousarray(theta, np.float64).ravel()
        pos = np.ascontiguousarray(pos, np.float64)
        rc = self.lib.vmo_eval(ctypes.byref(s), _ptr(theta), _ptr(pos), _ptr(grad), _ptr(lap),
                               _ptr(pgrad), _ptr(en))
        assert rc == 0, rc
        return grad.reshape(E, D), lap, pgrad.reshape(E, P), en

    def ratio(self, spec, theta, pos, k, xnew):
        s = spec.vmo()
        r = np.zeros(len(spec.elements))
        theta = np.ascontiguousarray(theta, np.float64).ravel()
        pos = np.ascontiguousarray(pos, np.float64)
        rc = self.lib.vmo_ratio(ctypes.byref(s), _ptr(theta), _ptr(pos), k, xnew, _ptr(r))
        assert rc == 0, rc
        return r

    def quantum_force(self, spec, theta, pos):
        s = spec.vmo()
        f = np.zeros(spec.D)
        theta = np.ascontiguousarray(theta, np.float64).ravel()
        rc = self.lib.vmo_quantum_force(ctypes.byref(s), _ptr(theta),
                                        _ptr(np.ascontiguousarray(pos, np.float64)), _ptr(f))
        assert rc == 0, rc
        return f

    def step_randoms(self, seed, walker, step, sampling):
        out = np.zeros(3)
        self.lib.vmo_step_randoms(seed, walker, step, sampling, _ptr(out))
        return out

    def initial_positions(self, seed, walker, D, normal, sd):
        out = np.zeros(D)
        self.lib.vmo_initial_positions(seed, walker, D, int(normal), sd, _ptr(out))
        return out

    def run(self, spec, theta, pos, fcache, steps, burn_in, iteration, batches, stream=None,
            seed=0, counter=None, want_steps=True, gpair=None):
        """pos, fcache: (W, D) arrays updated in place; gpair: (W, N, N) per-pair Pade
        gamma (updated in place) or None for fresh pair terms.  Returns dict of outputs."""
        s = spec.vmo()
        W, D = pos.shape
        E, P = len(spec.elements), spec.p_max
        NS = 9 + 2 * E * P
        sums = np.zeros((W, NS))
        acc = np.zeros((W, steps), np.uint8) if want_steps else None
        en = np.zeros((W, steps, 3)) if want_steps else None
        if counter is None:
            counter = np.zeros(W, np.uint64)
        theta = np.ascontiguousarray(theta, np.float64).ravel()
        st = None if stream is None else np.ascontiguousarray(stream, np.float64)
        rc = self.lib.vmo_run(ctypes.byref(s), _ptr(theta), W, _ptr(pos), _ptr(fcache),
                              _ptr(gpair), steps,
                              burn_in, iteration, batches, _ptr(st), seed, _ptr(counter),
                              _ptr(acc), _ptr(en), _ptr(sums))
        assert rc == 0, rc
        return {"sums": sums, "accepted": acc, "energies": en, "counter": counter}

    def blocking(self, x):
        x = np.ascontiguousarray(x, np.float64)
        mean = ctypes.c_double()
        var = self.lib.vmo_blocking(_ptr(x), len(x), ctypes.byref(mean))
        return mean.value, var


class RefHarness:
    """One reference System (one walker) at fixed positions with a replayed stream."""

    def __init__(self, spec, pos, theta=None, stream=None, path=REF_SO, text=None):
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.vmref_create.restype = ctypes.c_void_p
        L.vmref_create.argtypes = [ctypes.c_char_p, ctypes.c_void_p, ctypes.c_int,
                                   ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_long]
        for name in ("vmref_info", "vmref_get_params", "vmref_get_positions", "vmref_eval",
                     "vmref_reset"):
            getattr(L, name).argtypes = [ctypes.c_void_p] + [ctypes.c_void_p] * {
                "vmref_info": 1, "vmref_get_params": 1, "vmref_get_positions": 1,
                "vmref_eval": 4, "vmref_reset": 0}[name]
        L.vmref_move.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_void_p]
        L.vmref_steps.restype = ctypes.c_long
        L.vmref_steps.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
                                  ctypes.c_void_p, ctypes.c_void_p]
        L.vmref_iteration.restype = ctypes.c_long
        L.vmref_iteration.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.vmref_destroy.argtypes = [ctypes.c_void_p]
        self.spec = spec
        pos = np.ascontiguousarray(pos, np.float64)
        th = None if theta is None else np.ascontiguousarray(theta, np.float64).ravel()
        st = None if stream is None else np.ascontiguousarray(stream, np.float64).ravel()
        config = text if text is not None else spec.input_in()
        self.h = L.vmref_create(config.encode(), _ptr(pos), len(pos), _ptr(th),
                                0 if th is None else len(th), _ptr(st),
                                0 if st is None else len(st))
        assert self.h, "reference harness failed to build the system"
        info = np.zeros(8, np.int32)
        L.vmref_info(self.h, _ptr(info))
        self.N, self.d, self.D, self.E, self.P, self.batches, self.steps_wo, self.burn_in = map(
            int, info)

    def close(self):
        if self.h:
            self.lib.vmref_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()

    def params(self):
        out = np.zeros(self.E * self.P)
        self.lib.vmref_get_params(self.h, _ptr(out))
        return out.reshape(self.E, self.P)

    def positions(self):
        out = np.zeros(self.D)
        self.lib.vmref_get_positions(self.h, _ptr(out))
        return out

    def eval(self):
        grad, lap = np.zeros(self.E * self.D), np.zeros(self.E)
        pg, en = np.zeros(self.E * self.P), np.zeros(3)
        self.lib.vmref_eval(self.h, _ptr(grad), _ptr(lap), _ptr(pg), _ptr(en))
        return grad.reshape(self.E, self.D), lap, pg.reshape(self.E, self.P), en

    def move(self, k, xnew):
        r = np.zeros(self.E)
        self.lib.vmref_move(self.h, k, xnew, _ptr(r))
        return r

    def reset(self):
        self.lib.vmref_reset(self.h)

    def steps(self, n):
        acc = np.zeros(n, np.uint8)
        en = np.zeros((n, 3))
        pg = np.zeros((n, self.E, self.P))
        used = self.lib.vmref_steps(self.h, n, _ptr(acc), _ptr(en), _ptr(pg))
        return acc, en, pg, used

    def settings(self):
        """System's parsed settings (vmref_settings)."""
        L = self.lib
        L.vmref_settings.restype = ctypes.c_int
        L.vmref_settings.argtypes = [ctypes.c_void_p, ctypes.c_void_p]
        out = np.zeros(32)
        n = L.vmref_settings(self.h, _ptr(out))
        return out[:n]

    def trial_label(self):
        """System's trial wave-function label (vmref_trial_label)."""
        L = self.lib
        L.vmref_trial_label.restype = ctypes.c_long
        L.vmref_trial_label.argtypes = [ctypes.c_void_p, ctypes.c_char_p, ctypes.c_long]
        buf = ctypes.create_string_buffer(512)
        n = L.vmref_trial_label(self.h, buf, len(buf))
        assert n >= 0
        return buf.raw[:n].decode()

    def densities(self, n, bins, max_radius, radial=True, spatial=True, pair=True):
        """n steps counting the Sampler's densities after each (vmref_densities)."""
        L = self.lib
        L.vmref_densities.restype = ctypes.c_long
        L.vmref_densities.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        r = np.zeros(bins, np.int64) if radial else None
        sp = np.zeros((bins, bins), np.int64) if spatial else None
        pr = np.zeros((bins, bins), np.int64) if pair else None
        used = L.vmref_densities(self.h, n, bins, max_radius, _ptr(r), _ptr(sp), _ptr(pr))
        return r, sp, pr, used

    def simulation(self, max_iters, check=0, n_energies=5, tolerance=1e-6, adaptive=0, range_=10, additional=4,
                   additional_last=8):
        """System::runSimulation's loop with the convergence and adaptive-step tools
        (vmref_simulation): per iteration the sampled steps, the energy and the
        density-iteration flag."""
        L = self.lib
        L.vmref_simulation.restype = ctypes.c_long
        L.vmref_simulation.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
                                       ctypes.c_void_p]
        steps, energy, last = np.zeros(max_iters, np.int32), np.zeros(max_iters), np.zeros(max_iters, np.int32)
        n = L.vmref_simulation(self.h, check, n_energies, tolerance, adaptive, range_, additional, additional_last,
                               _ptr(steps), _ptr(energy), _ptr(last))
        return n, steps[:max(n, 0)], energy[:max(n, 0)], last[:max(n, 0)]

    def iteration(self, it):
        EP = self.E * self.P
        out = np.zeros(6 + 3 * EP)
        used = self.lib.vmref_iteration(self.h, it, _ptr(out))
        return {
            "energy": out[0], "std_error": out[1], "kinetic": out[2], "external": out[3],
            "interaction": out[4], "acceptance": out[5],
            "avg_grad": out[6:6 + EP].reshape(self.E, self.P),
            "avg_grad_e": out[6 + EP:6 + 2 * EP].reshape(self.E, self.P),
            "params": out[6 + 2 * EP:].reshape(self.E, self.P), "used": used,
        }


def load_cases(npz_path):
    """Group a golden .npz by case name: {name: {field: array}}."""
    z = np.load(npz_path, allow_pickle=False)
    cases = {}
    for key in z.files:
        name, field_ = key.split("/", 1)
        cases.setdefault(name, {})[field_] = z[key]
    return cases


def spec_from_case(c):
    """Rebuild the SystemSpec a golden case was generated with."""
    return SystemSpec(
        N=int(c["spec_N"]), d=int(c["spec_d"]), elements=tuple(int(e) for e in c["spec_elements"]),
        omega=float(c["spec_omega"]), Z=int(c["spec_Z"]), coulomb=bool(c["spec_coulomb"]),
        sampling=str(c["spec_sampling"]), step=float(c["spec_step"]), hidden=int(c["spec_hidden"]),
        atom=bool(c["spec_atom"]), sorting=bool(c["spec_sorting"]),
        optimization=str(c["spec_optimization"]), learning_rate=float(c["spec_learning_rate"]),
        num_steps=int(c["spec_num_steps"]),
        basis=str(c["spec_basis"]) if "spec_basis" in c else "hermite")
