"""Benchmark: walker-moves/s of the B200 engine on the N=56 quantum dot.

Workload (one "step" = one optimisation iteration of the whole walker population):
  2D quantum dot, N=56 electrons (two 28x28 Hermite Slater blocks) x Gaussian x
  Pade-Jastrow, omega=0.28, Coulomb, importance sampling dt=0.005, 16384 walkers x
  (20000 + 20 burn-in) single-coordinate moves per iteration, E_L and dlnPsi/dtheta
  sampled after every move (the reference's definition of a step), device-reduced
  sums, ADAM update.  Mixed precision (FP32 sweep, FP64 rebuild every refresh
  interval, compensated FP64 sums); an FP64 engine run of the same workload is
  reported beside it, and both arms are compared at equal sigma_E: one more iteration
  of each at the same parameters records every walker's local energy per step and
  blocks the series on the device (the reference's Blocker), and the time each arm
  needs to reach the same error bar follows from its iteration time and its sigma_E
  (sigma_E^2 falls as 1 / samples).  Synthetic: walker start positions from
  per-walker Philox streams, RandomNormal as in the reference.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl engine|reference]

N > 1: one process per GPU (torchrun), walkers per GPU fixed (weak scaling); the
only exchange per iteration is the NCCL all-reduce of the sampler totals
(vmachine_b200.distributed), plus the barrier and the max-over-ranks timing.
"""
import argparse
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import threading

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "N=56 dot walker-moves/s & E_L samples/s: mixed vs FP64 GPU at equal sigma_E"
UNIT = "walker-moves/s"
N_PART, OMEGA, DT = 56, 0.28, 0.005
REF_BIN = os.path.join(ROOT, "oracle", "_ref", "vmachine_ref")


def workload_text(walkers, steps_per_walker, precision, seed, refresh="auto"):
    return "\n".join([f"refreshInterval: {refresh}",
        f"numParticles: {N_PART}", "numDimensions: 2", "hamiltonian: harmonicOscillator",
        f"omega: {OMEGA}", "interactionStyle: coulomb",
        "waveFunctionElement: slaterDeterminant", "waveFunctionElement: gaussian",
        "waveFunctionElement: padeJastrow", "basis: hermite",
        "sampling: importanceSampling", f"stepLength: {DT}", "optimization: adam",
        "learningRate: 0.01", f"numSteps: {walkers * steps_per_walker}", "numIterations: 100",
        f"numWalkers: {walkers}", f"precision: {precision}", f"rng: MersenneTwister {seed}",
    ]) + "\n"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one launch of the mixed
# owner sweep on this workload's 16 384 walkers, from an ncu capture of a 448-step
# launch (not this run: the walker state is read and written once per launch, so the
# figure does not depend on the launch's step count)
SWEEP_TRAFFIC_BYTES = 225_813_760


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return None


def flops_per_step(N, d=2):
    """Algorithmic flops of one accepted move plus one E_L / dlnPsi sample in the
    engine's incremental, degree-factorised scheme (FMA = 2, MUL/ADD = 1,
    div/sqrt/exp = 1), term by term below: Hermite tables at the proposal, the ratio
    row contractions, the Sherman-Morrison update, the block's derivative refresh, the
    moved particle's pair terms, the kinetic sum and the scalar bookkeeping."""
    n = N // 2
    K = next(k for k in range(1, 12) if (k * (k + 1) // 2 if d == 2 else k * (k + 1) * (k + 2) // 6) == n)
    tables = d * 4 * (K - 1)                             # Hermite recurrence at one point
    ratio = tables + n * (2 * n + 2 * K)                 # S_j = phi(r_p') . inv[:, j], all j
    sm = 2 * n * n                                       # Sherman-Morrison rank-1 update
    per_orbital = 4 if d == 2 else 9
    deriv = n * (tables + per_orbital * n + 3 * d * (2 * K - 3))  # d ln det refresh of the block
    pairs = (N - 1) * (10 * d + 38)                      # Pade / Coulomb terms of the moved particle
    kinetic = 7 * N * d
    return ratio + sm + deriv + pairs + kinetic + 40


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms while running."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []

    def __enter__(self):
        if shutil.which("nvidia-smi"):
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.gpu}", f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["not sampled"]}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ---------------------------------------------------------------- reference arm

def reference_sample(cores, steps_per_proc, seed0=11):
    """Run `cores` concurrent single-rank reference processes on the workload's
    input.in (numSteps scaled down) and return aggregate walker-moves/s from the
    reference's own per-iteration CPU_time column."""
    if not os.path.exists(REF_BIN):
        return None, "oracle/_ref/vmachine_ref was not built"
    tmp = tempfile.mkdtemp(prefix="vmref_")
    procs = []
    for i in range(cores):
        d = os.path.join(tmp, f"p{i}")
        os.makedirs(d)
        txt = "\n".join([
            f"numParticles: {N_PART}", "numDimensions: 2", "hamiltonian: harmonicOscillator",
            f"omega: {OMEGA}", "interactionStyle: coulomb",
            "waveFunctionElement: slaterDeterminant", "waveFunctionElement: gaussian",
            "waveFunctionElement: padeJastrow", "basis: hermite",
            "sampling: importanceSampling", f"stepLength: {DT}", "optimization: adam",
            "learningRate: 0.01", f"numSteps: {steps_per_proc}", "numIterations: 2",
            f"rng: MersenneTwister {seed0 + i}", f"path: {d}/"]) + "\n"
        with open(os.path.join(d, "input.in"), "w") as f:
            f.write(txt)
        procs.append(subprocess.Popen([REF_BIN, "input.in"], cwd=d, stdout=subprocess.PIPE,
                                      stderr=subprocess.DEVNULL, text=True))
    rates = []
    for p in procs:
        out, _ = p.communicate(timeout=900)
        t = None
        for ln in out.splitlines():
            f = ln.split()
            if len(f) == 11 and f[0] == "1":
                t = float(f[-1])
        if t:
            rates.append((steps_per_proc + int(steps_per_proc * 0.001)) / t)
    shutil.rmtree(tmp, ignore_errors=True)
    if not rates:
        return None, "reference runs printed no iteration timing"
    return float(sum(rates)), None


def host_cores():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference_arm(args, rank):
    if rank != 0:
        return
    cores = host_cores()
    steps = args.ref_steps
    values = []
    for i in range(args.warmup + args.steps):
        v, err = reference_sample(cores, steps, seed0=11 + 1000 * i)
        if v is None:
            print(json.dumps({"impl": "reference", "unavailable": err}))
            return
        if i >= args.warmup:
            values.append(v)
    value = statistics.median(values)
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * (steps * cores) / value, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"2D quantum dot N={N_PART} omega={OMEGA}, Slater(Hermite) x "
                               "Gaussian x Pade, importance sampling dt=0.005, one walker per "
                               "process, E_L every move", "processes": cores,
                   "steps_per_process": steps},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                         "cpu_model": cpu_model(), "samples": values,
                         "sample": f"{cores} concurrent one-rank runs of the reference built "
                                   f"from its sources, {steps} moves each, CPU_time column"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))


# ---------------------------------------------------------------- engine arm

def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
        pg = dist
    return world, rank, local, pg


def barrier(pg, local):
    if pg is not None:
        import torch
        t = torch.zeros(1, device=f"cuda:{local}")
        pg.all_reduce(t)
        torch.cuda.synchronize(local)


def max_over_ranks(pg, local, v):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def run_engine_arm(args):
    world, rank, local, pg = dist_setup(args)
    from vmachine_b200 import Engine, measure_fma_peak
    from vmachine_b200 import distributed as vd
    W, spw = args.walkers, args.steps_per_walker
    # one population of world x W walkers, rank r holding walkers rW .. rW + W - 1 (their
    # random streams keyed by the population index: the shards are one engine's chains)
    seed = 1000
    shard = f"walkerOffset: {rank * W}\n"
    text = workload_text(W, spw, "mixed", seed, args.refresh_interval) + shard
    eng = Engine(text, device=local)
    eng.init_walkers(None, seed=seed)
    burn = eng.info.burn_in
    moves_per_step = W * (spw + burn)
    for it in range(args.warmup):
        vd.run_iteration(eng, it)
    barrier(pg, local)
    sweep_s, launches, sig, energies = 0.0, 0.0, [], []
    kernels = 0
    with ClockSampler(local) as clk:
        eng.stopwatch_start()
        for it in range(args.steps):
            # this iteration's kernels: a sweep and an FP64 re-inversion per launch of
            # refresh-interval steps, the accumulator reduction, two per-walker mean
            # gathers (the engine's spread estimate and the shard's copy) and the
            # re-inversion after the parameter step
            interval = eng.refresh_interval()
            n_launch = -(-(spw + burn) // interval) if interval > 0 else None
            kernels += 2 * n_launch + 4 if n_launch else 0
            a = vd.run_iteration(eng, args.warmup + it)  # all-reduce of the sums when N > 1
            sig.append(a.walker_std_error)
            energies.append((a.energy, a.walker_std_error))
        ms = eng.stopwatch_stop()
    # per-launch sweep timing of one more iteration (same work, not in the timed region)
    sums, _, _ = eng.sample(args.warmup + args.steps, spw + burn, burn)
    sweep_s, launches = sums.sweep_seconds, sums.sweep_launches
    max_drift, q99_drift = sums.max_drift, sums.q99_drift
    refresh_now = eng.refresh_interval()
    ms = max_over_ranks(pg, local, ms)
    total_moves = moves_per_step * args.steps * world
    value = total_moves / (ms * 1e-3)
    energy = a.energy

    # e2e through the C ABI with pinned host buffers: walkers uploaded, one iteration,
    # walkers read back, every step (each step's result is the next step's input)
    e2e = None
    if not args.no_e2e:
        import torch
        pinned = [torch.empty((eng.W, eng.D), dtype=torch.float64, pin_memory=True) for _ in range(2)]
        pos, nxt = (t.numpy() for t in pinned)
        eng.positions(out=pos)
        h2d = pos.nbytes + 8 * eng.E * eng.P
        d2h = pos.nbytes + 8 * 16
        barrier(pg, local)
        eng.stopwatch_start()
        for it in range(args.e2e_steps):
            eng.init_walkers(pos, seed=seed)
            vd.run_iteration(eng, 1000 + it)
            eng.positions(out=nxt)
            pos, nxt = nxt, pos
        e2e_ms = max_over_ranks(pg, local, eng.stopwatch_stop())
        e2e = {"value": moves_per_step * args.e2e_steps * world / (e2e_ms * 1e-3), "unit": UNIT,
               "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "path": "vmc_init_walkers(pinned host positions) + vmc_sample + vmc_apply_sums + "
                       "vmc_get_positions(into pinned host memory) per step"}

    # FP64 engine on the same workload (same walkers, fewer steps per iteration)
    fp64 = None
    if not args.no_fp64:
        # same walkers, seeds and schedule as the mixed arm: energies comparable
        eng64 = Engine(workload_text(W, spw, "fp64", seed) + shard, device=local)
        eng64.init_walkers(None, seed=seed)
        for it in range(args.warmup):
            vd.run_iteration(eng64, it)
        barrier(pg, local)
        eng64.stopwatch_start()
        e64 = []
        for it in range(args.fp64_steps):
            a64 = vd.run_iteration(eng64, args.warmup + it)
            e64.append((a64.energy, a64.walker_std_error))
        ms64 = max_over_ranks(pg, local, eng64.stopwatch_stop()) / args.fp64_steps
        mv64 = W * (spw + eng64.info.burn_in) * world
        fp64 = {"value": mv64 / (ms64 * 1e-3), "ms_per_step": ms64, "steps": args.fp64_steps,
                "energy": e64[-1][0], "sigma_e_walkers": e64[-1][1],
                "mixed_energy_same_iteration": energies[min(args.fp64_steps, args.steps) - 1][0],
                "mixed_sigma_same_iteration": energies[min(args.fp64_steps, args.steps) - 1][1]}
        if not args.no_sigma:
            # equal sigma_E: both arms start from the mixed arm's current walkers and
            # parameters (held fixed), make args.equil_passes sampling passes with their
            # own Philox streams (no optimiser step), then one recorded pass each (spw
            # sampled moves per walker), blocked on the device
            theta, pos = eng.parameters(), eng.positions()
            equil = {"mixed": [], "fp64": []}
            for name, e_ in (("mixed", eng), ("fp64", eng64)):
                e_.set_parameters(theta)
                e_.init_walkers(pos, seed=seed)
                for i in range(args.equil_passes):
                    s_, _, _ = e_.sample(0, spw + burn, burn)
                    equil[name].append(s_.energy / s_.n_samples)
            b32 = eng.blocking(spw + burn, burn)
            b64 = eng64.blocking(spw + burn, burn)
            t32, t64 = ms / args.steps * 1e-3, ms64 * 1e-3
            s32, s64 = b32.energy.std_error, b64.energy.std_error
            fp64["equal_sigma"] = {
                "blocking": "reference Blocker (automatic blocking, blocker.cpp) of every walker's "
                            "per-step E_L concatenated walker by walker, %d samples per walker; both "
                            "arms from the same walkers at the same fixed parameters, after %d "
                            "equilibration passes"
                            % (b32.samples_per_walker, args.equil_passes),
                "mixed": {"energy": b32.energy.mean, "sigma_e": s32, "sigma_e_walkers": b32.energy_walkers.std_error,
                          "s_per_iteration": t32},
                "fp64": {"energy": b64.energy.mean, "sigma_e": s64, "sigma_e_walkers": b64.energy_walkers.std_error,
                         "s_per_iteration": t64},
                "equilibration_pass_energies": equil,
                "energy_difference_in_error_bars": abs(b32.energy.mean - b64.energy.mean) / (s32 * s32 + s64 * s64) ** 0.5,
                "time_to_fp64_sigma_s": {"mixed": t32 * (s32 / s64) ** 2, "fp64": t64},
                "time_ratio": t64 / (t32 * (s32 / s64) ** 2),
            }
        eng64.close()

    # the heterogeneous multi-system batch (every rank takes part)
    batch = batch_line(args, pg, rank, local, world) if args.batch_iterations > 0 else None

    if rank != 0:
        if pg is not None:
            pg.destroy_process_group()
        return
    peak = measure_fma_peak(local, 1)
    fl = flops_per_step(N_PART)
    avg_launch = sweep_s / max(launches, 1)
    steps_per_launch = (spw + burn) / max(launches, 1)
    achieved = fl * W * steps_per_launch / avg_launch / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32 (f64 rebuild and sums)",
        "data": "synthetic (Philox RandomNormal starts, sigma = 1/omega)",
        "config": {"workload": f"2D quantum dot N={N_PART} omega={OMEGA}: Slater(Hermite, 2 x "
                               f"28x28) x Gaussian x Pade, Coulomb, importance sampling "
                               f"dt={DT}, E_L + dlnPsi every move, ADAM",
                   "walkers_per_gpu": W, "steps_per_walker": spw, "burn_in": burn,
                   "precision": "mixed", "refresh_interval": refresh_now,
                   "inverse_drift": {"max": max_drift, "q99": q99_drift},
                   "walkers_per_block": eng.info.walkers_per_block,
                   "kernel": ["runtime-flags", "compiled-in dot flags", "general"][eng.info.kernel_variant],
                   "sweep_form": {1: "staged", 2: "owner"}.get(eng.info.sweep_form),
                   "l2": "walker state %.0f MB per GPU > 126 MB L2, streamed every launch"
                         % (W * (eng.info.n_coords * 5 * 4 + 2 * 28 * 28 * 4 + 56 * 8 + 64) / 1e6)},
        "el_samples_per_s": value * spw / (spw + burn),
        "energy": energy, "sigma_e_walkers": sig[-1] if sig else None,
        "gpu_launches": int(kernels) if kernels else int(args.steps * (2 * launches + 4)),
        "roofline": {"bound": "fp32-pipe", "achieved": achieved, "peak": peak,
                     "unit": "TFLOP/s", "frac": achieved / peak if peak else None,
                     "traffic": SWEEP_TRAFFIC_BYTES,
                     "traffic_note": "stale capture: dram read + write bytes of one 448-step launch "
                                     "of the same kernel on the same 16 384 walkers under ncu, not "
                                     "measured in this run (the walker state is read and written once "
                                     "per launch whatever its length)",
                     "peak_source": "vmc_measure_fma_peak (FP32 FMA loop, this GPU, this run); "
                                    "MEASURED_PEAKS.json has no FP32 pipe figure",
                     "flops_per_move": fl,
                     "kernel": ("owner_sweep_kernel<float,7,reference flags>" if eng.info.sweep_form == 2
                                else "sweep_kernel<float,2,7>"),
                     "avg_launch_ms": avg_launch * 1e3},
    }
    if e2e:
        line["e2e"] = e2e
    if fp64:
        line["fp64"] = fp64
        line["mixed_over_fp64"] = value / fp64["value"]
    if args.learned > 0 and world == 1:
        from vmachine_b200.learned import compare
        line["learned"] = compare(budget_s=args.learned)
    if batch:
        line["batch"] = batch
    if not args.no_cpu_baseline and world == 1:
        cores = host_cores()
        v, err = reference_sample(cores, args.ref_steps)
        line["cpu_baseline"] = ({"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                                 "cpu_model": cpu_model(),
                                 "sample": f"{cores} concurrent one-rank reference runs, "
                                           f"{args.ref_steps} moves each"}
                                if v else {"value": None, "unavailable": err})
    line["clocks"] = clk.summary()
    print(json.dumps(line))
    eng.close()
    if pg is not None:
        pg.destroy_process_group()


def batch_line(args, pg, rank, local, world):
    """The heterogeneous workload (64 systems: 62 2D dots N = 2..56, He, Ne) through the
    multi-system batch: systems bin-packed by cost over the ranks, each rank one batch
    (persistent kernel, captured graph, tuned tile); walker-moves/s of the replayed
    iterations, device-timed, max over ranks."""
    from vmachine_b200.batch import mixed_systems, partition, run as batch_run
    texts, desc = mixed_systems(5, 2000)
    mine = partition(desc, world)[0][rank]
    r = batch_run(args.batch_iterations, texts=[texts[i] for i in mine], device=local)
    secs = max_over_ranks(pg, local, r["ms_per_iteration"] * 1e-3)
    moves = sum(desc[i]["walkers"] for i in range(len(desc))) * 2000.0
    return {"workload": "64 systems: 62 2D closed-shell dots N in {2,6,12,20,30,42,56}, omega ~ U[0.1, 1], "
                        "256-4096 walkers each; He and Ne atoms (hydrogen orbitals x SimpleJastrow, general "
                        "path: FP32 sweep, FP64 Slater inverse); mixed precision, 2000 steps per walker per "
                        "iteration, seed 5",
            "walker_moves_per_s": moves / secs, "ms_per_iteration": secs * 1e3, "systems_per_rank": len(mine),
            "tile": r["tile"], "graph_captures": r["graph_captures"], "replayed_iterations": r["replayed_iterations"],
            "tuning_ns_per_move": [t[3] for t in r["tuning"]], "scaling": "strong"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    # the mixed engine's FP64 re-inversion cadence settles in the warm-up: it starts at
    # 512 steps, the first passes from the starting distribution halve it to 256, and it
    # doubles per pass while the inverse drift stays small, reaching its 8 192-step cap
    # by the eighth pass
    ap.add_argument("--warmup", type=int, default=8)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--walkers", type=int, default=16384)
    ap.add_argument("--steps-per-walker", type=int, default=20000)
    ap.add_argument("--fp64-steps", type=int, default=5)
    ap.add_argument("--refresh-interval", default="auto")
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--ref-steps", type=int, default=60000)
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-sigma", action="store_true", help="skip the equal-sigma_E blocking runs")
    ap.add_argument("--equil-passes", type=int, default=3,
                    help="sampling passes at fixed parameters before the equal-sigma_E blocking runs")
    ap.add_argument("--batch-iterations", type=int, default=16,
                    help="iterations of the 64-system heterogeneous batch (0: skip)")
    ap.add_argument("--learned", type=float, default=0.0,
                    help="seconds of training per wave function for the MLP-vs-Pade comparison "
                         "at N=20 omega=0.5 (0: skip)")
    args = ap.parse_args()
    if args.impl == "reference":
        run_reference_arm(args, int(os.environ.get("RANK", "0")))
    else:
        run_engine_arm(args)


if __name__ == "__main__":
    main()
