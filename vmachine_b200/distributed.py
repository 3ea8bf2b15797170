"""Data-parallel VMC over several GPUs (one process per GPU, torch.distributed).

Walkers are independent Markov chains, so they shard across ranks with no
exchange during sampling.  A rank's engine holds a contiguous slice of one walker
population (`shard_text`: numWalkers and numSteps of the slice, `walkerOffset` = the
slice's first walker), and every walker's random streams are keyed by its index in
the whole population, so the shards together walk exactly the chains one engine
over all walkers would.

The one exchange per iteration replaces the reference's MPI_Reduce of the sampler
sums (src/sampler.cpp:111-187) and the MPI_Bcast of the parameters
(src/system.cpp:130-135): every rank all-reduces one packed vector (the 9
energy/acceptance sums, the sample and window counts, the 2 x n_elements x p_max
gradient sums, the per-walker energy means' moments, the status bits and an error
flag) and applies the same totals with vmc_apply_sums, so all ranks take the same
optimiser step.  A second all-reduce (minimum) gives every mixed-precision shard the
same FP64 refresh cadence for the next iteration.  A rank whose sampling pass fails
still takes part in both collectives, and then every rank raises the error.
"""
import re

import numpy as np

from .engine import Sums, VmcError

SUM_FIELDS = ("energy", "energy2", "kinetic", "kinetic2", "external", "external2",
              "interaction", "interaction2", "accepts", "n_samples", "n_window")
# walker status bits carried across ranks (vmc_sums.status: 1 NaN energy, 2 bad
# ratio, 4 singular block, 8 tensor-core wait gave up)
STATUS_BITS = (1, 2, 4, 8)
# tail of the payload: sum and sum of squares of the walkers' mean energies and their
# count, the status bits (0/1 each), the error flag and the error code
N_TAIL = 3 + len(STATUS_BITS) + 2


def shard_text(text, rank, world):
    """input.in of rank `rank`'s slice of the population that `text` configures:
    numWalkers and numSteps of the slice (the same steps per walker) and
    walkerOffset = its first walker.  Ranks take contiguous slices, the first
    W mod world ranks one walker more."""
    def value(key):
        m = re.search(rf"^\s*{key}\s*:\s*(\S+)", text, re.M)
        if not m:
            raise ValueError(f"{key} is needed to shard the population")
        return int(float(m.group(1)))
    W, steps = value("numWalkers"), value("numSteps")
    spw = steps // W
    base, extra = divmod(W, world)
    w_local = base + (1 if rank < extra else 0)
    offset = rank * base + min(rank, extra)
    out = re.sub(r"^\s*(numWalkers|numSteps|walkerOffset)\s*:.*\n?", "", text, flags=re.M)
    return out + f"numWalkers: {w_local}\nnumSteps: {spw * w_local}\nwalkerOffset: {offset}\n"


def pack(sums, grad_sum, egrad_sum, walker_means=None, error=None):
    """Sums + gradient sums (+ walker-mean moments, status bits, error) -> one
    float64 vector (the all-reduce payload)."""
    head = np.array([getattr(sums, f) for f in SUM_FIELDS], np.float64)
    m = np.asarray(walker_means if walker_means is not None else [], np.float64)
    status = int(getattr(sums, "status", 0))
    tail = [m.sum(), (m * m).sum(), float(m.size)] + [1.0 if status & b else 0.0 for b in STATUS_BITS]
    tail += [1.0, float(error)] if error is not None else [0.0, 0.0]
    return np.concatenate([head, np.ravel(grad_sum), np.ravel(egrad_sum), tail]).astype(np.float64)


def unpack(vec, n_elements, p_max):
    """-> (sums, grad_sum, egrad_sum, walker_std_error, error code or None)."""
    n = len(SUM_FIELDS)
    ep = n_elements * p_max
    if len(vec) != n + 2 * ep + N_TAIL:
        raise ValueError(f"payload has {len(vec)} values, expected {n + 2 * ep + N_TAIL}")
    s = Sums()
    for i, f in enumerate(SUM_FIELDS):
        setattr(s, f, float(vec[i]))
    g = np.array(vec[n:n + ep]).reshape(n_elements, p_max)
    ge = np.array(vec[n + ep:n + 2 * ep]).reshape(n_elements, p_max)
    t = vec[n + 2 * ep:]
    s1, s2, cnt = t[0], t[1], t[2]
    s.status = sum(b for b, on in zip(STATUS_BITS, t[3:3 + len(STATUS_BITS)]) if on > 0)
    # independent chains: spread of the walkers' mean energies over sqrt(walkers)
    wse = 0.0
    if cnt > 1:
        var = (s2 - s1 * s1 / cnt) / (cnt - 1)
        wse = float(np.sqrt(max(var, 0.0) / cnt))
    err = None
    if t[-2] > 0:
        err = int(round(t[-1] / t[-2])) if t[-2] == 1 else -3
    return s, g, ge, wse, err


def allreduce_sum(vec, group=None, op="sum"):
    """Sum (or minimum) of a float64 vector over the ranks of `group` (NCCL on the
    current GPU, or gloo on the CPU)."""
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        dev = torch.device("cuda", torch.cuda.current_device())
    else:
        dev = torch.device("cpu")
    t = torch.from_numpy(np.ascontiguousarray(vec, np.float64)).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM if op == "sum" else dist.ReduceOp.MIN, group=group)
    return t.cpu().numpy()


def world_size(group=None):
    try:
        import torch.distributed as dist
        return dist.get_world_size(group) if dist.is_initialized() else 1
    except Exception:
        return 1


def run_iteration(engine, iteration, group=None, allreduce=allreduce_sum):
    """One iteration of every rank's walker shard: sample, all-reduce the totals,
    apply them.  Returns the (global) averages, walker_std_error over all walkers."""
    info = engine.info
    steps = info.steps_per_walker + info.burn_in
    error = None
    try:
        sums, g, ge = engine.sample(iteration, steps, info.burn_in)
        means = engine.walker_energies()
    except VmcError as exc:
        sums, g, ge, means, error = Sums(), np.zeros((engine.E, engine.P)), np.zeros((engine.E, engine.P)), [], exc.code
    vec = pack(sums, g, ge, means, error)
    multi = world_size(group) > 1
    if multi:
        vec = allreduce(vec, group)
        if info.precision == 1:
            # every shard refreshes on the most cautious cadence any shard's drift test chose
            cadence = allreduce(np.array([float(engine.refresh_interval())]), group, op="min")
            if error is None:
                engine.set_refresh_interval(int(cadence[0]))
    total, gt, get, wse, err = unpack(vec, engine.E, engine.P)
    if err is not None:
        raise VmcError(err, "a rank's sampling pass failed" if error is None else f"sampling failed ({error})")
    avg = engine.apply_sums(total, gt, get)
    if isinstance(avg, dict):
        avg["walker_std_error"] = wse
    else:
        avg.walker_std_error = wse
    return avg
