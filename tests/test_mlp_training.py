"""What the learned MLP Jastrow gains, trained on the GPU by the engine's own
forward and backward kernels (N = 20, omega = 0.5 quantum dot).

- Training lowers the energy of the MLP wave function far below its untrained
  start (the network's output layers start at zero, so the untrained factor is the
  cusp term alone, with alpha = 1).
- At equal wall time the trained MLP's energy is not above the Pade-Jastrow's trained
  by the same engine by more than 3 sigma or 0.02 (0.02 %), whichever is larger: both
  frozen wave functions are evaluated
  by brute-force Metropolis in FP64 on fresh walkers with every walker's series
  blocked on the device (learned.evaluate_frozen), sigma the two blocked error bars
  in quadrature.  The gap and the variances of the local energy are printed.
Both factors run on the mixed-precision dot sweep.

The gap itself is not asserted: it depends on the training run.  Importance sampling
at dt = 0.01 leaves a few walkers stuck next to a node of the determinant, and the
MLP's gradient sums are accumulated with atomic additions, so two runs of the same
configuration part during training.  Runs of this test have ended with the MLP below
the Pade by 0.060 (18 sigma) and level with it (-0.0001, 0.0 sigma); in the second the
Pade itself ended 0.013 higher than in the first, so a run that perturbs only the MLP
could leave it a few sigma above.
"""
import math

import pytest

pytestmark = pytest.mark.gpu

BUDGET_S = 40.0


def test_trained_network_gains():
    from vmachine_b200 import Engine
    from vmachine_b200.learned import dot_config, evaluate, evaluate_frozen, train
    N, omega, W, steps = 20, 0.5, 2048, 800
    mlp_text = dot_config(N, omega, "mlpJastrow", W, steps, 3e-4)
    untrained = Engine(mlp_text)
    untrained.init_walkers(None, seed=7)
    e0, s0, _ = evaluate(untrained, 2000, burn_steps=1000)
    untrained.close()
    eng, hist = train(mlp_text, BUDGET_S)
    b_mlp = evaluate_frozen(eng, mlp_text, 2000, 1000)
    eng.close()
    pade_text = dot_config(N, omega, "padeJastrow", W, steps, 0.01)
    pade, phist = train(pade_text, BUDGET_S)
    b_pade = evaluate_frozen(pade, pade_text, 2000, 1000)
    pade.close()
    gap = b_pade["energy"] - b_mlp["energy"]
    sigma = math.hypot(b_pade["error"], b_mlp["error"])
    print(f"untrained {e0:.4f}+-{s0:.4f}  trained MLP {b_mlp['energy']:.4f}+-{b_mlp['error']:.4f} "
          f"var {b_mlp['variance']:.3f} ({len(hist)} iterations)  Pade {b_pade['energy']:.4f}+-{b_pade['error']:.4f} "
          f"var {b_pade['variance']:.3f} ({len(phist)} iterations)  gap {gap:.4f} = {gap / sigma:.1f} sigma")
    assert b_mlp["energy"] < e0 - 5 * (s0 + b_mlp["error"])
    assert gap > -max(3 * sigma, 0.02)
