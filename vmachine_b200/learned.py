"""What the learned MLP Jastrow gains over the Pade-Jastrow at equal wall time.

Two wave functions of the same 2D quantum dot, Slater(Hermite) x Gaussian x J with
J the Pade-Jastrow or the MLP Jastrow, are trained by the engine's own sampling and
ADAM steps (forward and backward kernels on the GPU) for the same wall-clock
budget each, then evaluated with their parameters frozen: every walker samples
`eval_steps` moves, and the energy's error bar is the spread of the walkers' mean
energies over sqrt(walkers) (the walkers are independent Markov chains).  The
variational principle decides: the lower energy at comparable error bars wins.
"""
import re
import time

import numpy as np

from .engine import Engine


def dot_config(N, omega, jastrow, walkers, steps, lr, dt=0.01, seed=7, extra=(), precision="mixed"):
    """Mixed precision runs both Jastrow factors on the FP32 dot sweep (the MLP's
    second layer on the tensor cores); fp64 runs the MLP on the general path."""
    lines = [f"numParticles: {N}", "numDimensions: 2", "hamiltonian: harmonicOscillator",
             f"omega: {omega!r}", "interactionStyle: coulomb",
             "waveFunctionElement: slaterDeterminant", "waveFunctionElement: gaussian",
             f"waveFunctionElement: {jastrow}", "basis: hermite", "sampling: importanceSampling",
             f"stepLength: {dt!r}", "optimization: adam", f"learningRate: {lr!r}",
             f"numSteps: {walkers * steps}", f"numWalkers: {walkers}", f"precision: {precision}",
             f"rng: MersenneTwister {seed}", "compat: corrected"]
    return "\n".join(lines + list(extra)) + "\n"


def train(text, budget_s, max_iterations=100000, seed=7):
    """Optimisation iterations until the wall-clock budget is spent; returns the
    engine (walkers equilibrated, parameters trained) and the energy history."""
    eng = Engine(text)
    eng.init_walkers(None, seed=seed)
    t0, hist = time.time(), []
    for it in range(max_iterations):
        a = eng.run_iteration(it)
        hist.append((time.time() - t0, a.energy, a.std_error))
        if hist[-1][0] >= budget_s:
            break
    return eng, hist


def evaluate(eng, eval_steps, burn_steps=200):
    """Energy of the frozen wave function: mean over walkers of each walker's mean
    local energy over eval_steps moves, with the standard error over walkers."""
    info = eng.info
    eng.sample(10 ** 6, burn_steps + 1, burn_steps)  # re-equilibrate after the last update
    eng.sample(10 ** 6, eval_steps + 1, 1)
    e = eng.walker_energies()
    return float(np.mean(e)), float(np.std(e, ddof=1) / np.sqrt(len(e))), int(info.n_walkers)


def evaluate_blocked(eng, eval_steps, burn_steps=200, fresh_seed=None):
    """The frozen wave function with every walker's local-energy series blocked on the
    device (vmc_blocking: the reference's Blocker per walker, include/block/blocker.cpp):
    the energy with its independent-chains error bar (each walker's own blocked
    variance of its mean, summed over walkers / W^2, so a walker that sits near a node
    for the whole pass weighs by its own fluctuation, not by its distance from the
    others), the concatenated-series Blocker result, and the variance of the local
    energy, the variational principle's second criterion.

    fresh_seed: start from new walkers drawn from the configured initial state with
    this seed (then burn_steps of equilibration) instead of the training's walkers.  A
    walker that importance sampling has left stuck next to a node of the determinant
    (a persistent configuration: its drift overshoots and nearly every move is
    rejected, with local energies of thousands) would otherwise carry over from
    training and dominate both the mean and the variance.
    flagged_walkers counts walkers whose status bits were set during the evaluation
    (2: a NaN acceptance weight, the mark of such a configuration)."""
    if fresh_seed is not None:
        eng.init_walkers(None, seed=fresh_seed)
    eng.sample(10 ** 6, burn_steps + 1, burn_steps)
    b = eng.blocking(eval_steps + 1, 1)
    s, _, _ = eng.sample(10 ** 6, eval_steps + 1, 1)
    var = s.energy2 / s.n_samples - (s.energy / s.n_samples) ** 2
    e = eng.walker_energies()
    return {"energy": b.energy_walkers.mean, "error": b.energy_walkers.std_error,
            "energy_blocker": b.energy.mean, "error_blocker": b.energy.std_error,
            "variance": float(var), "samples_per_walker": int(b.samples_per_walker),
            "walker_median": float(np.median(e)), "walker_max_deviation": float(np.max(np.abs(e - np.median(e)))),
            "flagged_walkers": int(np.count_nonzero(eng.status()))}


def evaluate_frozen(eng, text, eval_steps=4000, burn_steps=2000, step_length=1.0, seed=1007):
    """The trained parameters of `eng` evaluated by brute-force Metropolis in FP64 on
    fresh walkers (a second engine from `text` with sampling: bruteForce,
    stepLength: step_length, precision: fp64), every walker's series blocked
    (evaluate_blocked).  The expectation value of a frozen wave function does not
    depend on the sampler, and brute-force moves carry no drift: importance sampling
    at dt = 0.01 leaves a few walkers stuck next to a node of the determinant (the
    drift, about 2 / distance there, throws every proposal far off, and nearly every
    move is rejected), and such a walker's mean local energy, in the thousands, would
    dominate the estimate and its variance."""
    t = re.sub(r"^sampling:.*$", "sampling: bruteForce", text, flags=re.M)
    t = re.sub(r"^driftLimit:.*\n?", "", t, flags=re.M)
    t = re.sub(r"^stepLength:.*$", f"stepLength: {step_length!r}", t, flags=re.M)
    t = re.sub(r"^precision:.*$", "precision: fp64", t, flags=re.M)
    ev = Engine(t)
    try:
        ev.set_parameters(eng.parameters())
        return evaluate_blocked(ev, eval_steps, burn_steps, fresh_seed=seed)
    finally:
        ev.close()


def compare(N=20, omega=0.5, walkers=4096, steps=800, budget_s=120.0, eval_steps=4000,
            lr_pade=0.01, lr_mlp=3e-4, seed=7, mlp_iterations=None, eval_burn=2000, drift_limit=0.0):
    """Pade against MLP Jastrow at equal wall time: both train for budget_s seconds,
    or, with mlp_iterations, the MLP trains for that many iterations and the Pade
    factor for the MLP's wall time; then each frozen wave function is evaluated, on
    the training's walkers ("energy", "error": walker means) and blocked on fresh
    walkers after eval_burn steps of equilibration ("blocked"), and by brute-force
    Metropolis in FP64 on fresh walkers ("frozen", evaluate_frozen).  drift_limit > 0
    trains both with the corrected mode's drift limiter (driftLimit)."""
    out = {"system": f"2D dot N={N} omega={omega}", "walkers": walkers, "steps_per_iteration": steps,
           "drift_limit": drift_limit,
           "budget_s": budget_s, "eval_steps_per_walker": eval_steps}
    runs = (("pade", "padeJastrow", lr_pade), ("mlp", "mlpJastrow", lr_mlp))
    if mlp_iterations:
        runs = runs[::-1]
    for name, jastrow, lr in runs:
        text = dot_config(N, omega, jastrow, walkers, steps, lr, seed=seed,
                          extra=[f"driftLimit: {drift_limit!r}"] if drift_limit > 0 else ())
        if name == "mlp" and mlp_iterations:
            eng, hist = train(text, float("inf"), max_iterations=mlp_iterations, seed=seed)
            budget_s = hist[-1][0]
            out["budget_s"] = budget_s
        else:
            eng, hist = train(text, budget_s, seed=seed)
        energy, err, W = evaluate(eng, eval_steps)
        out[name] = {"iterations": len(hist), "train_seconds": hist[-1][0], "lr": lr,
                     "last_iteration_energy": hist[-1][1], "energy": energy, "error": err,
                     "blocked": evaluate_blocked(eng, eval_steps, eval_burn, fresh_seed=seed + 1000),
                     "frozen": evaluate_frozen(eng, text, eval_steps, eval_burn, seed=seed + 1000)}
        eng.close()
    d = out["pade"]["energy"] - out["mlp"]["energy"]
    out["gain"] = d
    out["gain_sigma"] = d / np.hypot(out["pade"]["error"], out["mlp"]["error"])
    bp, bm = out["pade"]["blocked"], out["mlp"]["blocked"]
    out["gain_blocked"] = bp["energy"] - bm["energy"]
    out["gain_blocked_sigma"] = out["gain_blocked"] / np.hypot(bp["error"], bm["error"])
    out["variance_ratio"] = bm["variance"] / bp["variance"]
    fp, fm = out["pade"]["frozen"], out["mlp"]["frozen"]
    out["gain_frozen"] = fp["energy"] - fm["energy"]
    out["gain_frozen_sigma"] = out["gain_frozen"] / np.hypot(fp["error"], fm["error"])
    out["variance_ratio_frozen"] = fm["variance"] / fp["variance"]
    return out


def sweep_speed(walkers=8192, steps=100, N=20, omega=0.5, tensor_cores=True, iterations=2, precision="mixed"):
    """Walker-moves per second of the MLP-Jastrow sweep (sampling and the backward
    kernel included) over `iterations` optimisation iterations after one warm-up.
    precision mixed: the FP32 dot sweep (tensor cores required); fp64: the general path."""
    if not tensor_cores:
        precision = "fp64"
    text = dot_config(N, omega, "mlpJastrow", walkers, steps, 3e-4, precision=precision,
                      extra=[f"mlpTensorCores: {'true' if tensor_cores else 'false'}"])
    eng = Engine(text)
    try:
        eng.init_walkers(None, seed=1)
        eng.run_iteration(0)
        eng.stopwatch_start()
        for it in range(iterations):
            a = eng.run_iteration(1 + it)
        ms = eng.stopwatch_stop()
        moves = iterations * walkers * (eng.info.steps_per_walker + eng.info.burn_in)
        return {"walkers": walkers, "steps_per_walker": steps, "tensor_cores": tensor_cores, "precision": precision,
                "ms_per_iteration": ms / iterations, "walker_moves_per_s": moves / (ms * 1e-3),
                "energy": a.energy, "status": int(np.bitwise_or.reduce(eng.status()))}
    finally:
        eng.close()


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(prog="python -m vmachine_b200.learned")
    sub = ap.add_subparsers(dest="cmd", required=True)
    s = sub.add_parser("speed", help="sweep throughput of the MLP-Jastrow wave function")
    s.add_argument("--walkers", type=int, default=8192)
    s.add_argument("--steps", type=int, default=100)
    s.add_argument("--cuda-cores", action="store_true", help="second layer on the CUDA cores (general path)")
    s.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                   help="mixed: the FP32 dot sweep; fp64: the general path")
    c = sub.add_parser("compare", help="MLP against Pade at equal wall time")
    c.add_argument("--budget", type=float, default=120.0)
    c.add_argument("--walkers", type=int, default=4096)
    c.add_argument("--steps", type=int, default=800, help="steps per walker per iteration")
    c.add_argument("--iterations", type=int, default=0,
                   help="train the MLP for this many iterations and the Pade factor for the same wall time")
    c.add_argument("--lr-mlp", type=float, default=3e-4)
    c.add_argument("--lr-pade", type=float, default=0.01)
    c.add_argument("--drift-limit", type=float, default=0.0, help="train with the corrected mode's drift limiter")
    a = ap.parse_args(argv)
    if a.cmd == "speed":
        print(json.dumps(sweep_speed(a.walkers, a.steps, tensor_cores=not a.cuda_cores, precision=a.precision)))
    else:
        print(json.dumps(compare(walkers=a.walkers, steps=a.steps, budget_s=a.budget, lr_mlp=a.lr_mlp,
                                 lr_pade=a.lr_pade, mlp_iterations=a.iterations or None,
                                 drift_limit=a.drift_limit)))


if __name__ == "__main__":
    main()
