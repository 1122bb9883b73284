"""The design loop (GPU forward + steady adjoint + sensitivity, CPU MMA
update) on a small channel: the MMA iterates stay in [0, 1], the volume
constraint is driven to its bound, and the objective history is finite."""
import numpy as np
import pytest

from implexity_b200 import workloads
from implexity_b200.optimize import DesignLoop, c5_initial_design, c5_problem

pytestmark = pytest.mark.gpu


def test_design_loop_small_channel(gpu_lib):
    shape = (24, 12, 12)
    loop = DesignLoop(c5_problem(shape, forward_steps=400), workloads.objective_weights(), volume_fraction=0.4)
    try:
        out = loop.run(c5_initial_design(shape, 0), iterations=4)
    finally:
        loop.close()
    h = out["history"]
    raw = out["final_design"]
    assert len(h) == 4
    assert np.all(np.isfinite([r["objective"] for r in h]))
    assert raw.min() >= 0.0 and raw.max() <= 1.0
    # the initial design (~0.52) violates the 0.4 volume bound; MMA moves toward it
    assert h[-1]["volume_fraction"] < h[0]["volume_fraction"]
    assert all(r["adjoint_iterations"] > 0 for r in h)


def test_design_loop_gcmma_small_channel(gpu_lib):
    """The GCMMA path of the loop: every trial design is evaluated by a forward
    solve, the accepted approximations are conservative (or the inner loop
    ran out), and the volume moves toward its bound."""
    shape = (24, 12, 12)
    loop = DesignLoop(c5_problem(shape, forward_steps=400), workloads.objective_weights(), volume_fraction=0.4,
                      gcmma=True)
    try:
        out = loop.run(c5_initial_design(shape, 0), iterations=3)
    finally:
        loop.close()
    h = out["history"]
    assert len(h) == 3
    assert np.all(np.isfinite([r["objective"] for r in h]))
    assert loop.trial_evaluations == sum(r["gcmma_inner"] + 1 for r in h)
    assert all(r["conservative"] or r["gcmma_inner"] == 15 for r in h)
    assert h[-1]["volume_fraction"] < h[0]["volume_fraction"]
