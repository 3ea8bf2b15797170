"""Heterogeneous multi-system workloads for the batch engine (vmachine_b200.Batch).

`mixed_systems` builds the 64-system workload the batch is measured on: 62 2D
closed-shell quantum dots with N in {2, 6, 12, 20, 30, 42, 56} (cycled), omega
drawn from U[0.1, 1] and a walker count from U{256..4096}, Slater(Hermite) x
Gaussian x Pade-Jastrow with importance sampling; plus the helium and neon atoms
(Z = 2 and 10; Slater determinants of hydrogen orbitals, 1x1 and 5x5 blocks, times
the SimpleJastrow factor) on the general path, in the workload's precision (mixed:
the atoms' FP32 sweep with the Slater inverse in FP64, re-inverted in FP64 after each
launch).  Everything is drawn from one seed, so the workload is reproducible.

`partition` spreads systems over ranks by cost (walkers x steps x work per step,
longest first onto the least loaded rank); the systems are independent, so ranks
exchange nothing while they run.

    python -m vmachine_b200.batch --iterations 16 [--alone]   # tune, capture, replay; JSON line
"""
import numpy as np

DOT_N = (2, 6, 12, 20, 30, 42, 56)


def dot_text(N, omega, walkers, steps, precision="mixed", seed=1, lr=0.01, compat="corrected"):
    dt = 0.01 if N <= 20 else 0.005
    return "\n".join([
        f"numParticles: {N}", "numDimensions: 2", "hamiltonian: harmonicOscillator", f"omega: {omega!r}",
        "interactionStyle: coulomb", "waveFunctionElement: slaterDeterminant",
        "waveFunctionElement: gaussian", "waveFunctionElement: padeJastrow", "basis: hermite",
        "sampling: importanceSampling", f"stepLength: {dt!r}", "optimization: adam", f"learningRate: {lr!r}",
        f"numSteps: {walkers * steps}", f"numWalkers: {walkers}", f"precision: {precision}",
        f"seed: {seed}", f"compat: {compat}"]) + "\n"


def atom_text(Z, walkers, steps, seed=1, lr=0.01, compat="corrected", precision="fp64"):
    return "\n".join([
        f"numParticles: {Z}", "numDimensions: 3", f"atomicNumber: {Z}", "hamiltonian: atomicNucleus",
        "interactionStyle: coulomb", "waveFunctionElement: slaterDeterminant",
        "waveFunctionElement: simpleJastrow", "basis: hydrogenOrbital", "sampling: importanceSampling",
        "stepLength: 0.01", "optimization: adam", f"learningRate: {lr!r}", f"numSteps: {walkers * steps}",
        f"numWalkers: {walkers}", f"precision: {precision}", f"seed: {seed}", f"compat: {compat}"]) + "\n"


def mixed_systems(seed=5, steps=2000, n_dots=62, precision="mixed", atoms=True, max_walkers=4096):
    """(texts, descriptions): the dots then He and Ne."""
    rng = np.random.default_rng(seed)
    texts, desc = [], []
    for i in range(n_dots):
        N = DOT_N[i % len(DOT_N)]
        omega = float(np.round(rng.uniform(0.1, 1.0), 6))
        W = int(rng.integers(256, max_walkers + 1))
        texts.append(dot_text(N, omega, W, steps, precision, seed=1000 + i))
        desc.append({"kind": "dot", "N": N, "omega": omega, "walkers": W})
    if atoms:
        for j, Z in enumerate((2, 10)):
            W = int(rng.integers(256, max_walkers + 1))
            texts.append(atom_text(Z, W, steps, seed=2000 + j, precision=precision))
            desc.append({"kind": "atom", "Z": Z, "N": Z, "walkers": W})
    return texts, desc


def step_cost(d):
    """Work per walker-step, for partitioning (the dot sweep's flop count; atoms as
    FP64 general-path steps)."""
    N = d["N"]
    if d["kind"] == "atom":
        return 8.0 * (N * N * 16 + (N // 2) ** 2 * 8 + N * 3 * 32)
    n = N // 2
    K = next(k for k in range(1, 12) if k * (k + 1) // 2 == n)
    tables = 8 * (K - 1)
    return (tables + n * (2 * n + 2 * K) + 2 * n * n + n * (tables + 4 * n + 6 * (2 * K - 3)) +
            (N - 1) * 58 + 14 * N + 40)


def partition(desc, world, steps=1):
    """Systems per rank: longest-processing-time-first onto the least loaded rank."""
    cost = [d["walkers"] * steps * step_cost(d) for d in desc]
    order = sorted(range(len(desc)), key=lambda i: -cost[i])
    load = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += cost[i]
    return [sorted(p) for p in parts], load


def run(iterations=12, seed=5, steps=2000, device=0, texts=None):
    """Iterate the mixed workload; walker-moves/s of the replayed (tuned) iterations."""
    import time

    from .engine import Batch
    if texts is None:
        texts, _ = mixed_systems(seed, steps)
    with Batch(texts, device=device) as b:
        b.init_walkers()
        per_it = []
        t0 = time.time()
        for it in range(iterations):
            b.run_iteration(it)
            i = b.info()
            per_it.append((i.graph_replay, i.seconds, i.sweep_seconds, i.walker_moves, i.rounds))
        wall = time.time() - t0
        info = b.info()
        replayed = [p for p in per_it if p[0]]
        secs = sum(p[1] for p in replayed)
        moves = sum(p[3] for p in replayed)
        sweep = sum(p[2] for p in replayed)
        sums = b.last_sums()
        return {"systems": len(texts), "walkers": int(info.n_walkers),
                "walker_moves_per_iteration": per_it[-1][3],
                "tile": {"walkers_per_block": info.walkers_per_block, "walkers_per_item": info.walkers_per_item,
                         "grid": info.grid},
                "tuning": b.tuning(), "graph_captures": info.graph_captures,
                "replayed_iterations": len(replayed),
                "walker_moves_per_s": moves / secs if secs > 0 else None,
                "sweep_walker_moves_per_s": moves / sweep if sweep > 0 else None,
                "ms_per_iteration": 1e3 * secs / max(1, len(replayed)),
                "wall_s": wall, "status": int(np.bitwise_or.reduce([s.status for s in sums])),
                "statuses": [int(s.status) for s in sums],
                "energies": [a.energy / a.n_samples for a in sums]}


def alone(texts, iterations=3, device=0):
    """The same systems one after another, each on its own engine and kernels (the
    way without a batch): device time of the iterations after the first, summed."""
    from .engine import Engine
    total_ms, moves = 0.0, 0.0
    for t in texts:
        with Engine(t, device=device) as e:
            e.init_walkers(None, seed=e.info.steps_per_walker)
            e.run_iteration(0)
            e.stopwatch_start()
            for it in range(1, iterations):
                e.run_iteration(it)
            total_ms += e.stopwatch_stop()
            moves += (iterations - 1) * e.W * (e.info.steps_per_walker + e.info.burn_in)
    return {"walker_moves_per_s": moves / (total_ms * 1e-3), "ms_per_iteration": total_ms / (iterations - 1)}


def main(argv=None):
    import argparse
    import json
    ap = argparse.ArgumentParser(prog="python -m vmachine_b200.batch")
    ap.add_argument("--iterations", type=int, default=12)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--seed", type=int, default=5)
    ap.add_argument("--alone", action="store_true", help="also time the systems one by one")
    a = ap.parse_args(argv)
    texts, desc = mixed_systems(a.seed, a.steps)
    r = run(a.iterations, a.seed, a.steps, texts=texts)
    r["flagged"] = [dict(d, status=st, energy=en) for d, st, en in zip(desc, r.pop("statuses"), r.pop("energies"))
                    if st]
    if a.alone:
        r["alone"] = alone(texts)
        r["batch_over_alone"] = r["walker_moves_per_s"] / r["alone"]["walker_moves_per_s"]
    print(json.dumps(r))


if __name__ == "__main__":
    main()
