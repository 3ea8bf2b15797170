"""Data-parallel VMC over several GPUs (one process per GPU, torch.distributed).

Walkers are independent Markov chains, so they shard across ranks with no
exchange during sampling.  The one exchange per iteration replaces the
reference's MPI_Reduce of the sampler sums (src/sampler.cpp:111-187) and the
MPI_Bcast of the parameters (src/system.cpp:130-135): every rank all-reduces the
packed totals (9 energy/acceptance sums, the sample and window counts, and the
2 x n_elements x p_max gradient sums) and applies the same totals with
vmc_apply_sums, so all ranks take the same optimiser step and stay in lockstep.
"""
import numpy as np

from .engine import Sums

SUM_FIELDS = ("energy", "energy2", "kinetic", "kinetic2", "external", "external2",
              "interaction", "interaction2", "accepts", "n_samples", "n_window")


def pack(sums, grad_sum, egrad_sum):
    """Sums + gradient sums -> one float64 vector (the all-reduce payload)."""
    head = np.array([getattr(sums, f) for f in SUM_FIELDS], np.float64)
    return np.concatenate([head, np.ravel(grad_sum), np.ravel(egrad_sum)]).astype(np.float64)


def unpack(vec, n_elements, p_max):
    n = len(SUM_FIELDS)
    ep = n_elements * p_max
    if len(vec) != n + 2 * ep:
        raise ValueError(f"payload has {len(vec)} values, expected {n + 2 * ep}")
    s = Sums()
    for i, f in enumerate(SUM_FIELDS):
        setattr(s, f, float(vec[i]))
    g = np.array(vec[n:n + ep]).reshape(n_elements, p_max)
    ge = np.array(vec[n + ep:n + 2 * ep]).reshape(n_elements, p_max)
    return s, g, ge


def allreduce_sum(vec, group=None):
    """Sum a float64 vector over the ranks of `group` (NCCL on the current GPU, or
    gloo on the CPU)."""
    import torch
    import torch.distributed as dist
    if dist.get_backend(group) == "nccl":
        dev = torch.device("cuda", torch.cuda.current_device())
    else:
        dev = torch.device("cpu")
    t = torch.from_numpy(np.ascontiguousarray(vec, np.float64)).to(dev)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t.cpu().numpy()


def world_size(group=None):
    try:
        import torch.distributed as dist
        return dist.get_world_size(group) if dist.is_initialized() else 1
    except Exception:
        return 1


def run_iteration(engine, iteration, group=None, allreduce=allreduce_sum):
    """One iteration of every rank's walker shard: sample, all-reduce the totals,
    apply them.  Returns the (global) averages."""
    info = engine.info
    steps = info.steps_per_walker + info.burn_in
    sums, g, ge = engine.sample(iteration, steps, info.burn_in)
    vec = pack(sums, g, ge)
    if world_size(group) > 1:
        vec = allreduce(vec, group)
    total, gt, get = unpack(vec, engine.E, engine.P)
    return engine.apply_sums(total, gt, get)
