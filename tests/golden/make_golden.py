"""Generate the golden fixtures in tests/golden/ from the reference itself.

Runs in the build container only: it drives oracle/_ref/libvmref.so, which
oracle/Makefile (`make ref`) compiles from the reference's own C++ sources.  The
fixtures it writes are committed, so the tests that use them need neither the
reference nor its build.

    python tests/golden/make_golden.py            # rewrites tests/golden/*.npz
    python tests/golden/make_golden.py hydrogen   # only hydrogen_orbitals.npz
    python tests/golden/make_golden.py hydrogen_sj   # only hydrogen_simplejastrow.npz
    python tests/golden/make_golden.py weights    # only weights_format.npz
    python tests/golden/make_golden.py densities  # only densities.npz
    python tests/golden/make_golden.py schedules  # only schedules.npz

Every input is seeded synthetic data: walker positions ~ N(0, 1/sqrt(omega)),
replayed uniforms/normals from numpy's PCG64 with fixed seeds.
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
from oracle_bind import (GAUSSIAN, HYDROGENLIKE, PADE, RBMGAUSSIAN, RBMPRODUCT,  # noqa: E402
                         SIMPLEJASTROW, SLATER, RefHarness, SystemSpec)

G, S, P = GAUSSIAN, SLATER, PADE


def spec_fields(spec):
    return dict(N=spec.N, d=spec.d, elements=np.array(spec.elements), omega=spec.omega, Z=spec.Z,
                coulomb=int(spec.coulomb), sampling=spec.sampling, step=spec.step,
                hidden=spec.hidden, atom=int(spec.atom), sorting=int(spec.sorting),
                optimization=spec.optimization, learning_rate=spec.learning_rate,
                num_steps=spec.num_steps, basis=spec.basis, config=spec.input_in())


EVAL_CASES = [
    ("n2_gauss_pade", SystemSpec(N=2, elements=(G, P)), 1.0, [[1.0], [0.5]]),
    ("n2_gauss_noint", SystemSpec(N=2, elements=(G,), coulomb=False), 1.0, None),
    ("n6_slater_gauss_pade", SystemSpec(N=6, elements=(S, G, P)), 1.0, [[0], [0.9], [0.7]]),
    ("n12_slater_gauss_pade", SystemSpec(N=12, elements=(S, G, P)), 1.0, None),
    ("n20_w05_slater_gauss_pade", SystemSpec(N=20, omega=0.5, elements=(S, G, P)),
     1 / np.sqrt(0.5), [[0], [1.02], [0.41]]),
    ("n30_w05_slater_gauss_pade", SystemSpec(N=30, omega=0.5, elements=(S, G, P)),
     1 / np.sqrt(0.5), None),
    ("n42_w028_slater_gauss_pade", SystemSpec(N=42, omega=0.28, elements=(S, G, P)),
     1 / np.sqrt(0.28), None),
    ("n56_w028_slater_gauss_pade", SystemSpec(N=56, omega=0.28, elements=(S, G, P)),
     1 / np.sqrt(0.28), [[0], [1.0], [0.35]]),
    ("n8_3d_slater_gauss_pade", SystemSpec(N=8, d=3, elements=(S, G, P)), 1.0, None),
    ("n6_slater_gauss_simplejastrow", SystemSpec(N=6, elements=(S, G, SIMPLEJASTROW)), 1.0,
     "random"),
    ("n2_rbm", SystemSpec(N=2, elements=(RBMGAUSSIAN, RBMPRODUCT), hidden=2), 1.0, "random"),
    ("n2_rbm_sorted", SystemSpec(N=2, elements=(RBMGAUSSIAN, RBMPRODUCT), hidden=3,
                                 sorting=True), 1.0, "random"),
    ("he_hydrogenlike_pade", SystemSpec(N=2, d=3, elements=(HYDROGENLIKE, P), atom=True, Z=2),
     1.0, [[1.0], [0.4]]),
]

CHAIN_CASES = [
    ("n2_gauss_pade_is", SystemSpec(N=2, elements=(G, P), step=0.1), 600),
    ("n2_gauss_pade_bf", SystemSpec(N=2, elements=(G, P), sampling="bruteForce", step=0.1), 600),
    ("n2_gauss_noint_bf", SystemSpec(N=2, elements=(G,), coulomb=False, sampling="bruteForce"),
     300),
    ("n6_slater_gauss_pade_is", SystemSpec(N=6, elements=(S, G, P), step=0.05), 500),
    ("n12_slater_gauss_pade_bf", SystemSpec(N=12, elements=(S, G, P), sampling="bruteForce"),
     400),
    ("n20_w05_slater_gauss_pade_is", SystemSpec(N=20, omega=0.5, elements=(S, G, P), step=0.01),
     400),
    ("n56_w028_slater_gauss_pade_is", SystemSpec(N=56, omega=0.28, elements=(S, G, P),
                                                 step=0.005), 250),
    ("n6_slater_gauss_simplejastrow_is", SystemSpec(N=6, elements=(S, G, SIMPLEJASTROW)), 400),
    ("n2_rbm_sorted_is", SystemSpec(N=2, elements=(RBMGAUSSIAN, RBMPRODUCT), sorting=True), 400),
    ("he_hydrogenlike_pade_is", SystemSpec(N=2, d=3, elements=(HYDROGENLIKE, P), atom=True, Z=2,
                                           step=0.05), 400),
]

ITER_CASES = [
    ("n2_gauss_pade_adam", SystemSpec(N=2, elements=(G, P), num_steps=2000, learning_rate=0.1),
     4),
    ("n2_gauss_pade_gd", SystemSpec(N=2, elements=(G, P), optimization="gd", num_steps=2000,
                                    learning_rate=0.1, sampling="bruteForce"), 4),
    ("n2_gauss_pade_sgd_momentum", SystemSpec(N=2, elements=(G, P), optimization="sgd 0.5 0.3",
                                              num_steps=2000, learning_rate=0.05), 4),
    ("n6_slater_gauss_pade_adam", SystemSpec(N=6, elements=(S, G, P), num_steps=1500,
                                             step=0.05), 3),
]


# Slater determinants of hydrogen orbitals (hydrogenorbital.cpp): He, Be, Ne, Mg, Ar.
# Written to their own file with their own seed, so the fixtures above stay as they are.
H_ORB = dict(d=3, atom=True, basis="hydrogenOrbital")
HYDROGEN_EVAL = [
    ("he_horb_pade", SystemSpec(N=2, Z=2, elements=(S, P), **H_ORB), 1.0, [[0], [0.4]]),
    ("be_horb_pade", SystemSpec(N=4, Z=4, elements=(S, P), **H_ORB), 1.0, [[0], [0.35]]),
    ("ne_horb_pade", SystemSpec(N=10, Z=10, elements=(S, P), **H_ORB), 0.6, [[0], [0.3]]),
    ("ne_horb_noint", SystemSpec(N=10, Z=10, elements=(S,), coulomb=False, **H_ORB), 0.6, None),
    ("mg_horb_pade", SystemSpec(N=12, Z=12, elements=(S, P), **H_ORB), 0.8, [[0], [0.3]]),
    ("ar_horb_pade", SystemSpec(N=18, Z=18, elements=(S, P), **H_ORB), 0.8, [[0], [0.25]]),
]
HYDROGEN_CHAINS = [
    ("he_horb_pade_is", SystemSpec(N=2, Z=2, elements=(S, P), step=0.05, **H_ORB), 300),
    ("ne_horb_pade_is", SystemSpec(N=10, Z=10, elements=(S, P), step=0.01, **H_ORB), 300),
    ("ne_horb_pade_bf", SystemSpec(N=10, Z=10, elements=(S, P), sampling="bruteForce", step=0.02,
                                   **H_ORB), 300),
]


def theta_for(spec, how, rng):
    E = len(spec.elements)
    Pm = spec.p_max
    if how is None:
        return None
    if isinstance(how, str):
        return rng.uniform(-0.3, 0.3, (E, Pm)) + 0.5
    th = np.zeros((E, Pm))
    for e, row in enumerate(how):
        th[e, :len(row)] = row
    return th


def make_eval(rng, cases=EVAL_CASES):
    out = {}
    for name, spec, scale, how in cases:
        theta = theta_for(spec, how, rng)
        rec = {k: [] for k in ("pos", "grad", "lap", "pgrad", "energies", "k", "xnew", "ratios",
                               "grad2", "lap2", "pgrad2", "energies2")}
        th_used = None
        for t in range(3):
            pos = rng.normal(0.0, scale, spec.D)
            R = RefHarness(spec, pos, theta)
            th_used = R.params()
            g, lap, pg, en = R.eval()
            k = int(rng.integers(spec.D))
            xn = pos[k] + rng.normal(0.0, 0.3)
            ratios = R.move(k, xn)
            g2, lap2, pg2, en2 = R.eval()
            R.close()
            for key, val in zip(rec, (pos, g, lap, pg, en, k, xn, ratios, g2, lap2, pg2, en2)):
                rec[key].append(val)
        arrays = {f"{name}/{k}": np.array(v) for k, v in rec.items()}
        arrays[f"{name}/theta"] = th_used
        for k, v in spec_fields(spec).items():
            arrays[f"{name}/spec_{k}"] = np.array(v)
        out.update(arrays)
    return out


def make_stream(spec, steps, rng):
    st = np.empty((steps, 3))
    st[:, 0] = rng.random(steps)
    st[:, 1] = rng.normal(size=steps) if spec.sampling == "importanceSampling" else rng.random(steps)
    st[:, 2] = rng.random(steps)
    return st


def make_chains(rng, cases=CHAIN_CASES):
    out = {}
    for name, spec, steps in cases:
        scale = 1.0 / np.sqrt(spec.omega) if not spec.atom else 1.0
        pos = rng.normal(0.0, scale, spec.D)
        stream = make_stream(spec, steps, rng)
        R = RefHarness(spec, pos, None, stream)
        theta = R.params()
        acc, en, pg, used = R.steps(steps)
        assert used == 3 * steps, (name, used)
        final = R.positions()
        R.close()
        for k, v in dict(pos=pos, theta=theta, stream=stream, accepted=acc, energies=en,
                         pgrads=pg, final_pos=final).items():
            out[f"{name}/{k}"] = v
        for k, v in spec_fields(spec).items():
            out[f"{name}/spec_{k}"] = np.array(v)
    return out


def make_iterations(rng):
    out = {}
    for name, spec, iters in ITER_CASES:
        pos = rng.normal(0.0, 1.0, spec.D)
        R0 = RefHarness(spec, pos)
        per_iter = R0.steps_wo + R0.burn_in
        R0.close()
        stream = make_stream(spec, per_iter * iters, rng)
        R = RefHarness(spec, pos, None, stream)
        theta0 = R.params()
        recs = [R.iteration(it) for it in range(iters)]
        R.close()
        out[f"{name}/pos"] = pos
        out[f"{name}/theta0"] = theta0
        out[f"{name}/stream"] = stream
        out[f"{name}/burn_in"] = np.array(R.burn_in)
        out[f"{name}/steps_wo"] = np.array(R.steps_wo)
        out[f"{name}/batches"] = np.array(R.batches)
        for key in ("energy", "std_error", "kinetic", "external", "interaction", "acceptance",
                    "avg_grad", "avg_grad_e", "params"):
            out[f"{name}/{key}"] = np.array([r[key] for r in recs])
        for k, v in spec_fields(spec).items():
            out[f"{name}/spec_{k}"] = np.array(v)
    return out


def make_blocking(rng):
    import ctypes
    from oracle_bind import REF_SO
    lib = ctypes.CDLL(REF_SO)
    lib.vmref_blocking.argtypes = [ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p]
    out = {}
    for i, (n, phi) in enumerate([(2 ** 11, 0.0), (2 ** 13, 0.9), (2 ** 14, 0.99)]):
        x = np.empty(n)
        e = rng.normal(size=n)
        x[0] = e[0]
        for t in range(1, n):
            x[t] = phi * x[t - 1] + e[t]
        x += 3.0
        res = np.zeros(2)
        lib.vmref_blocking(x.ctypes.data_as(ctypes.c_void_p), n, res.ctypes.data_as(ctypes.c_void_p))
        out[f"series{i}/x"] = x
        out[f"series{i}/mean"] = res[0]
        out[f"series{i}/std_error"] = res[1]
    return out


def make_weights(rng):
    """Parameter files as the reference writes them (Sampler::printParametersToFile:
    the matrix through Eigen's default stream format, then endl)."""
    import ctypes
    from oracle_bind import REF_SO
    lib = ctypes.CDLL(REF_SO)
    lib.vmref_format_weights.restype = ctypes.c_long
    lib.vmref_format_weights.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_char_p,
                                         ctypes.c_long]
    mats = [np.array([[0.0], [1.02029717], [0.35]]), np.array([[1.0], [0.5]]),
            rng.normal(size=(2, 3)), rng.normal(scale=40.0, size=(3, 4)),
            np.array([[1e-7, -123456.789, 0.0], [1.5e10, -2.5e-12, 7.0]]),
            rng.normal(scale=0.3, size=(3, 36)), -np.abs(rng.normal(size=(4, 5))) * 1e-3]
    out = {}
    for i, m in enumerate(mats):
        m = np.ascontiguousarray(m, np.float64)
        buf = ctypes.create_string_buffer(1 << 16)
        n = lib.vmref_format_weights(m.ctypes.data_as(ctypes.c_void_p), m.shape[0], m.shape[1], buf, len(buf))
        assert 0 < n < len(buf)
        out[f"matrix{i}/theta"] = m
        out[f"matrix{i}/text"] = np.array(buf.value.decode())
    return out


# The same atoms with a SimpleJastrow factor (the general path's compiled atom form),
# in a file of their own so the fixtures above stay as they are.
HYDROGEN_SJ_EVAL = [
    ("he_horb_sj", SystemSpec(N=2, Z=2, elements=(S, SIMPLEJASTROW), **H_ORB), 1.0, "random"),
    ("ne_horb_sj", SystemSpec(N=10, Z=10, elements=(S, SIMPLEJASTROW), **H_ORB), 0.6, "random"),
    ("ne_horb_pade_sj", SystemSpec(N=10, Z=10, elements=(S, P, SIMPLEJASTROW), **H_ORB), 0.6, "random"),
]
HYDROGEN_SJ_CHAINS = [
    ("he_horb_sj_is", SystemSpec(N=2, Z=2, elements=(S, SIMPLEJASTROW), step=0.05, **H_ORB), 300),
    ("ne_horb_sj_is", SystemSpec(N=10, Z=10, elements=(S, SIMPLEJASTROW), step=0.01, **H_ORB), 300),
    ("ne_horb_sj_bf", SystemSpec(N=10, Z=10, elements=(S, SIMPLEJASTROW), sampling="bruteForce", step=0.02,
                                 **H_ORB), 300),
]


def make_hydrogen_sj():
    rng = np.random.default_rng(20261206)
    out = make_eval(rng, HYDROGEN_SJ_EVAL)
    out.update({f"chain_{k}": v for k, v in make_chains(rng, HYDROGEN_SJ_CHAINS).items()})
    np.savez_compressed(os.path.join(HERE, "hydrogen_simplejastrow.npz"), **out)


DENSITY_CASES = [
    # atoms: the Metropolis keeps System's radial vector current (the atomic Hamiltonian
    # needs it), so all three of the reference's densities count the walker as it moves
    ("he_horb_sj", SystemSpec(N=2, Z=2, elements=(S, SIMPLEJASTROW), step=0.05, **H_ORB), 3, 500, 40, 4.0),
    ("be_horb_pade", SystemSpec(N=4, Z=4, elements=(S, P), step=0.02, **H_ORB), 2, 400, 30, 5.0),
    # a dot: only the spatial density (the reference's radial densities of a dot count the
    # initial radii, its radial vector not being updated: elementoperation.cpp:130-170)
    ("n6_slater_gauss_pade", SystemSpec(N=6, elements=(S, G, P), step=0.05), 3, 500, 40, 4.0),
]


def make_densities():
    """Per case, walkers each with its own replayed stream through the reference's
    Metropolis, densities counted after every step (no burn-in), summed over walkers."""
    rng = np.random.default_rng(20261207)
    out = {}
    for name, spec, walkers, steps, bins, rmax in DENSITY_CASES:
        pos = np.stack([rng.normal(0.0, 1.0, spec.D) for _ in range(walkers)])
        streams = np.stack([make_stream(spec, steps, rng) for _ in range(walkers)])
        radial = np.zeros(bins, np.int64)
        spatial = np.zeros((bins, bins), np.int64)
        pair = np.zeros((bins, bins), np.int64)
        # one parameter set for every walker (random initial weights would otherwise be
        # drawn from each walker's own stream)
        R0 = RefHarness(spec, pos[0], None, streams[0])
        theta = R0.params()
        R0.close()
        for w in range(walkers):
            R = RefHarness(spec, pos[w], theta, streams[w])
            r, sp, pr, used = R.densities(steps, bins, rmax)
            assert used == 3 * steps, (name, used)
            R.close()
            radial += r
            spatial += sp
            pair += pr
        for k, v in dict(pos=pos, stream=streams, theta=theta, bins=np.array(bins), max_radius=np.array(rmax),
                         radial=radial, spatial=spatial, pair=pair).items():
            out[f"{name}/{k}"] = v
        for k, v in spec_fields(spec).items():
            out[f"{name}/spec_{k}"] = np.array(v)
    np.savez_compressed(os.path.join(HERE, "densities.npz"), **out)


SCHEDULE_TOOLS = dict(check=1, n_energies=3, tolerance=0.05, adaptive=1, range_=3, additional=1,
                      additional_last=2)
SCHEDULE_CASES = [
    # converges at iteration 2 (|E_0 - E_2| < 0.05), so `normal` = 3, the density
    # iteration is 6 (x4 steps), 3-5 and the ones after it take x2 steps; the loop goes on
    # to numIterations (system.cpp:93 has no exit at the last iteration)
    ("n2_converge", SystemSpec(N=2, elements=(G, P), step=0.1, sampling="bruteForce", num_steps=2000,
                               extra=["numIterations: 14", "checkConvergence: true", "numberOfEnergies: 3",
                                      "tolerance: 0.05", "applyAdaptiveSteps: true", "rangeOfAdaptiveSteps: 3",
                                      "additionalSteps: 1", "additionalStepsLastIter: 2"]), 14),
    # no convergence (tolerance 0): the last iteration is numIterations - 1
    ("n2_no_converge", SystemSpec(N=2, elements=(G, P), step=0.1, sampling="bruteForce", num_steps=2000,
                                  extra=["numIterations: 8", "checkConvergence: true", "numberOfEnergies: 3",
                                         "tolerance: 0.0", "applyAdaptiveSteps: true", "rangeOfAdaptiveSteps: 3",
                                         "additionalSteps: 1", "additionalStepsLastIter: 2"]), 8),
]


def make_schedules():
    """System::runSimulation's schedule on one walker with a replayed stream: per
    iteration the sampled steps, the energy and the density iteration, under the
    convergence check and adaptive steps."""
    rng = np.random.default_rng(20261208)
    out = {}
    for name, spec, iters in SCHEDULE_CASES:
        tools = dict(SCHEDULE_TOOLS)
        if name == "n2_no_converge":
            tools["tolerance"] = 0.0
        pos = rng.normal(0.0, 1.0, spec.D)
        stream = make_stream(spec, 2000 * 4 * iters + 100, rng)
        R = RefHarness(spec, pos, None, stream)
        theta = R.params()
        n, steps, energy, last = R.simulation(iters, **tools)
        R.close()
        assert n == iters, (name, n)
        for k, v in dict(pos=pos, stream=stream, theta=theta, steps=steps, energy=energy, last=last).items():
            out[f"{name}/{k}"] = v
        for k, v in spec_fields(spec).items():
            out[f"{name}/spec_{k}"] = np.array(v)
        out[f"{name}/extra"] = np.array("\n".join(spec.extra))
    np.savez_compressed(os.path.join(HERE, "schedules.npz"), **out)


def make_hydrogen():
    rng = np.random.default_rng(20261204)
    out = make_eval(rng, HYDROGEN_EVAL)
    out.update({f"chain_{k}": v for k, v in make_chains(rng, HYDROGEN_CHAINS).items()})
    np.savez_compressed(os.path.join(HERE, "hydrogen_orbitals.npz"), **out)


def main():
    if sys.argv[1:] == ["hydrogen"]:
        make_hydrogen()
        return
    if sys.argv[1:] == ["hydrogen_sj"]:
        make_hydrogen_sj()
        return
    if sys.argv[1:] == ["schedules"]:
        make_schedules()
        return
    if sys.argv[1:] == ["densities"]:
        make_densities()
        return
    if sys.argv[1:] == ["weights"]:
        np.savez_compressed(os.path.join(HERE, "weights_format.npz"),
                            **make_weights(np.random.default_rng(20261205)))
        return
    make_hydrogen()
    make_hydrogen_sj()
    make_densities()
    make_schedules()
    rng = np.random.default_rng(20261203)
    np.savez_compressed(os.path.join(HERE, "eval_fixed.npz"), **make_eval(rng))
    np.savez_compressed(os.path.join(HERE, "chains.npz"), **make_chains(rng))
    np.savez_compressed(os.path.join(HERE, "iterations.npz"), **make_iterations(rng))
    np.savez_compressed(os.path.join(HERE, "blocking.npz"), **make_blocking(rng))
    np.savez_compressed(os.path.join(HERE, "weights_format.npz"), **make_weights(np.random.default_rng(20261205)))
    for f in sorted(os.listdir(HERE)):
        if f.endswith(".npz"):
            print(f, os.path.getsize(os.path.join(HERE, f)))


if __name__ == "__main__":
    main()
