"""Several walkers per warp for the small dots.

A walker of a small dot fills few of a warp's 32 lanes (one per orbital row, partner
or coordinate group), so the production sweep gives each walker an 8-lane quarter
(N <= 6) or a 16-lane half (N = 12 to 30) of the warp; N = 42 and 56 keep one walker
per warp by default (the owner form, test_owner_sweep_gpu.py) and take two on request
in the staged form (`walkersPerWarp: 2`, rows of the 21 x 21
and 28 x 28 inverse blocks in two passes).  The walkers see the same random numbers and the same
arithmetic either way, so the iterations of a population swept several per warp
equal those swept one per warp (`walkersPerWarp: 1`).  A population of 37 leaves
the last warp with one walker.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def run(text, iterations):
    from vmachine_b200 import Engine
    out = []
    with Engine(text, device=0) as e:
        e.init_walkers(None, seed=3)
        info = e.info
        for it in range(iterations):
            a = e.run_iteration(it)
            out.append((a.energy, a.kinetic, a.interaction, a.acceptance, e.parameters().copy()))
        pos = e.positions()
    return info, out, pos


@pytest.mark.parametrize("N,omega,per_warp", [(2, 1.0, 4), (6, 0.5, 4), (6, 0.5, 2), (12, 0.8, 2), (20, 0.5, 2),
                                                (30, 0.6, 2), (42, 0.4, 2), (56, 0.28, 2)])
@pytest.mark.parametrize("precision", ["fp64", "mixed"])
@pytest.mark.parametrize("compat", ["reference", "corrected"])
def test_walkers_per_warp_equal_one(N, omega, per_warp, precision, compat):
    from vmachine_b200.batch import dot_text
    # both arms in the staged form (one walker per warp would otherwise take the owner
    # form at N = 42 and 56; tests/test_owner_sweep_gpu.py compares the two forms)
    text = dot_text(N, omega, 37, 300, precision, seed=11, compat=compat) + "sweepForm: staged\n"
    i2, two, p2 = run(text + f"walkersPerWarp: {per_warp}\n", 3)
    i1, one, p1 = run(text + "walkersPerWarp: 1\n", 3)
    assert i2.walkers_per_warp == per_warp and i1.walkers_per_warp == 1
    tol = 1e-12 if precision == "fp64" else 1e-5
    for (e2, k2, v2, a2, t2), (e1, k1, v1, a1, t1) in zip(two, one):
        assert abs(e2 - e1) <= tol * abs(e1), (e2, e1)
        assert abs(k2 - k1) <= tol * abs(k1)
        assert abs(v2 - v1) <= tol * max(abs(v1), 1e-300)
        assert abs(a2 - a1) <= 1e-3
        assert np.allclose(t2, t1, rtol=tol, atol=0)
    assert np.allclose(p2, p1, rtol=tol * 10, atol=tol * 10)


def test_walkers_per_warp_selection():
    """Four per warp for the compiled-in dots of N <= 6, two for N = 12 to 30, one for
    larger dots; four for the atoms of at most 4 electrons, one for the rest of the
    general path."""
    from vmachine_b200 import Engine
    from vmachine_b200.batch import atom_text, dot_text
    for N, expect in ((2, 4), (6, 4), (12, 2), (20, 2), (30, 2), (42, 1), (56, 1)):
        with Engine(dot_text(N, 0.5, 64, 10, "mixed"), device=0) as e:
            assert e.info.walkers_per_warp == expect, N
    # atoms on the general path: four per warp for He (at most 4 electrons; its
    # replayed chains against the oracle run in this form), one for Ne
    with Engine(atom_text(2, 64, 10), device=0) as e:
        assert e.info.walkers_per_warp == 4
    with Engine(atom_text(10, 64, 10), device=0) as e:
        assert e.info.walkers_per_warp == 1
