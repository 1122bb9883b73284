"""Central finite differences of the GPU objective along seeded Gaussian
directions against the adjoint directional derivative (the check of
implexity-ad's gradcheck.rs:218-291, restated in implexity_b200.gradcheck).

FP32 forward state: J carries ~1e-7 relative rounding noise while a design
step h moves it by ~1e-3 h relative on this grid, so the step is 1e-2 on the
raw design (central-difference truncation ~h^2) and the bar is 1e-2 relative
per direction for the exact (horizon) gradient.
"""
import numpy as np
import pytest

from implexity_b200 import LbmSolver, normalize, workloads
from implexity_b200.gradcheck import directional_check

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("lattice", ["D3Q19", "D3Q27"])
def test_directional_fd_matches_horizon_adjoint(gpu_lib, lattice):
    shape = (16, 10, 8)
    prob = workloads.channel_problem(shape=shape, steps=200, collision="trt", lattice=lattice)
    norm = normalize(prob)
    raw = workloads.uniform_design(shape, 3)
    w = workloads.objective_weights()
    editable = (np.asarray(norm.design_region, bool) & ~np.asarray(norm.solid_mask, bool)).reshape(shape)
    with LbmSolver(norm) as s:
        s.set_design(raw)
        s.forward()
        g, _ = s.gradient(w, mode="horizon", checkpoint_every=50)
        res = directional_check(s, raw, w, g, editable, count=4, seed=11, step=1e-2)
    for r in res:
        assert r.rel_error < 1e-2, r
