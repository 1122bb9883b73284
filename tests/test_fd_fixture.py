"""The finite-difference check at the specified step: central differences at
step 1e-4 along 8 seeded Gaussian directions (gradcheck.rs:218-232, taken
along a direction; directions of implexity_b200.gradcheck.directions, seeds
0..7) of J = pressure drop + viscous dissipation after 5000 steps of the 32^3
channel, computed with the FP64 oracle as the forward
(tests/golden/make_scale_fixtures.py).  An FP32 forward cannot take this step
itself: its ~1e-7 relative rounding of J is comparable to what a 1e-4 design
step changes.

The GPU's horizon gradient (the exact discrete gradient of J) and its steady
gradient (the fixed-point adjoint; the 32^3 forward is converged after 5000
steps) must give the same directional derivatives within 1e-4 relative.
"""
from pathlib import Path

import numpy as np
import pytest

from implexity_b200 import LbmSolver, normalize, workloads
from implexity_b200.gradcheck import directions

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden"


def test_oracle_fd_at_step_1e4_matches_gpu_adjoint(gpu_lib):
    import make_scale_fixtures as m

    fx = dict(np.load(GOLDEN / "fd_channel32_trt.npz"))
    shape = tuple(int(v) for v in fx["shape"])
    raw = workloads.uniform_design(shape, int(fx["design_seed"]))
    norm = normalize(m.fd_problem())
    editable = (np.asarray(norm.design_region, bool) & ~np.asarray(norm.solid_mask, bool)).reshape(shape)
    w = workloads.objective_weights()
    with LbmSolver(norm) as s:
        s.set_design(raw)
        s.forward()
        J = float(np.dot(w, s.responses()))
        g_h, _ = s.gradient(w, mode="horizon", checkpoint_every=100)
        s.forward()  # the horizon adjoint's recomputation leaves the state elsewhere
        g_s, rep = s.gradient(w, mode="steady", tolerance=1e-10)
    assert rep.converged
    J_ref = float(fx["objective"])
    # FP32 collision arithmetic: the coherent-rounding floor of the steady
    # pressure (tests/test_scale_parity.py); FP64 collision arithmetic: the
    # specification's 1e-6
    assert abs(J - J_ref) <= 1e-5 * abs(J_ref)
    prob64 = m.fd_problem()
    prob64["solver_options"]["collision_arithmetic"] = "float64"
    with LbmSolver(normalize(prob64)) as s64:
        s64.set_design(raw)
        s64.forward()
        J64 = float(np.dot(w, s64.responses()))
    assert abs(J64 - J_ref) <= 1e-6 * abs(J_ref), abs(J64 - J_ref) / abs(J_ref)
    dirs = list(directions(raw, editable, len(fx["seeds"]), int(fx["seeds"][0]), float(fx["fd_step"])))
    for k, (seed, d) in enumerate(dirs):
        assert seed == int(fx["seeds"][k])
        fd = float(fx["fd"][k])
        for name, g in (("horizon", g_h), ("steady", g_s)):
            ad = float(np.dot(g.ravel(), d.ravel()))
            rel = abs(ad - fd) / abs(fd)
            assert rel < 1e-4, (name, seed, ad, fd, rel)
