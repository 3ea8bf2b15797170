"""Host side of the multi-system batch without a GPU: the mixed workload's
systems parse and pass the engine's support checks (they fail only at the CUDA
step here), the batch rejects what it cannot hold before touching CUDA, and the
systems split over ranks by cost with no exchange (two gloo ranks)."""
import ctypes
import os

import numpy as np
import pytest
import torch.distributed as dist
import torch.multiprocessing as mp

from vmachine_b200.batch import mixed_systems, partition, step_cost

E_CONFIG, E_UNSUPPORTED, E_CUDA, E_ARG = -1, -2, -3, -4


def test_mixed_workload_shape():
    texts, desc = mixed_systems(seed=5)
    assert len(texts) == 64
    dots = [d for d in desc if d["kind"] == "dot"]
    assert len(dots) == 62 and {d["N"] for d in dots} == {2, 6, 12, 20, 30, 42, 56}
    assert all(0.1 <= d["omega"] <= 1.0 and 256 <= d["walkers"] <= 4096 for d in dots)
    assert [d["Z"] for d in desc if d["kind"] == "atom"] == [2, 10]
    assert mixed_systems(seed=5) == (texts, desc)
    assert mixed_systems(seed=6)[1] != desc


def test_every_system_is_accepted():
    from vmachine_b200 import library
    lib = library()
    for t in mixed_systems(seed=5)[0]:
        h = ctypes.c_void_p()
        rc = lib.vmc_create(t.encode(), None, ctypes.byref(h))
        if rc == 0:
            lib.vmc_destroy(h)
        assert rc in (0, E_CUDA), (rc, lib.vmc_last_error(), t)


@pytest.mark.parametrize("texts,code", [
    ([], E_ARG),
    (["numParticles: 2\nbogusKey: 1\n"], E_CONFIG),
    (["numParticles: 2\nhamiltonian: harmonicOscillator\nwaveFunctionElement: gaussian\n"] * 65, E_ARG),
])
def test_batch_rejects(texts, code):
    from vmachine_b200 import library
    lib = library()
    arr = (ctypes.c_char_p * max(1, len(texts)))(*[t.encode() for t in texts])
    h = ctypes.c_void_p()
    rc = lib.vmc_batch_create(arr, len(texts), None, ctypes.byref(h))
    assert rc == code, lib.vmc_last_error()
    assert not h.value
    # the device slot is free again: a second attempt fails the same way, not with "exists"
    assert lib.vmc_batch_create(arr, len(texts), None, ctypes.byref(h)) == code


def test_partition_balances_cost():
    _, desc = mixed_systems(seed=5)
    for world in (1, 2, 4, 8):
        parts, load = partition(desc, world)
        assert sorted(i for p in parts for i in p) == list(range(len(desc)))
        total = sum(d["walkers"] * step_cost(d) for d in desc)
        biggest = max(d["walkers"] * step_cost(d) for d in desc)
        assert max(load) <= total / world + biggest  # LPT bound


def _rank(rank, world, port, out):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    _, desc = mixed_systems(seed=5)
    mine, _ = partition(desc, world)
    got = [None] * world
    dist.all_gather_object(got, mine[rank])
    if rank == 0:
        out.put(got)
    dist.destroy_process_group()


def test_two_ranks_take_disjoint_systems():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    procs = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = q.get(timeout=120)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    a, b = set(got[0]), set(got[1])
    assert not (a & b) and len(a | b) == 64
