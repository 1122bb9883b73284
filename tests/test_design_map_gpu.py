"""The reference's default design map on the GPU: conic filter (DesignMap::new,
design.rs:107-171), tanh projection and fixed/solid overrides (map,
design.rs:199-216) and their transpose (vjp, design.rs:219-243), through the
C-ABI, against the golden fixtures and the FP64 oracle.

Cases:
  the reference's own problem template (provider.rs:74-90; 4x6x4 BGK,
  periodic x/z, body force, conic filter 1.5 mm, projection beta 2), whose
  golden file holds an independent numpy restatement's trajectory, responses
  and complex-step gradient (tests/golden/make_golden.py);
  a channel with a conic filter of radius 2 cells, projection beta 8, solid
  cells inside the design region and a block of the design region taken out
  (random fixed values there; the port planes stay fixed fluid).

Tolerances: phi 1e-6 absolute, alpha 1e-5 relative, state 1e-5 relative (max
norm), responses 1e-5 relative, horizon gradient 1e-4 relative L2.
"""
import numpy as np
import pytest

from implexity_b200 import LbmSolver, normalize, workloads
from oracle.oracle import Oracle

from _problems import golden_problem, load_golden
from test_gpu_parity import rel_l2, rel_max

pytestmark = pytest.mark.gpu


def test_reference_template_through_the_abi(gpu_lib):
    g = load_golden("template_bgk")
    norm = normalize(golden_problem("template_bgk"))
    o = Oracle(norm)
    with LbmSolver(norm) as s:
        s.set_design(g["raw"])
        phi, alpha = s.design()
        assert np.max(np.abs(phi.ravel() - g["phi"])) < 1e-6
        assert rel_max(alpha, g["alpha"]) < 1e-5
        d = s.forward()
        assert d.admitted
        f = s.populations()
        assert rel_max(f, g["final"]) < 1e-5
        r = s.responses()
        for k in (0, 3, 4, 5, 6, 7):
            assert abs(r[k] - g["responses"][k]) <= 1e-5 * max(abs(g["responses"][k]), 1e-300), k
        for k in (1, 2):  # transverse mean velocities against the axial one
            assert abs(r[k] - g["responses"][k]) <= 1e-5 * abs(g["responses"][0]), k
        grad, _ = s.gradient(g["weights"], mode="horizon", checkpoint_every=3)
    cells = g["fd_cells"]
    assert rel_l2(grad.ravel()[cells], g["fd_grad"]) < 1e-4
    g_ref, _, _, st = o.gradient(g["raw"], g["weights"], mode="horizon", K=3)
    assert st == 0
    assert rel_l2(grad, g_ref) < 1e-4


def conic_channel(lattice="D3Q19"):
    shape = (20, 12, 10)
    nx, ny, nz = shape
    solid = np.zeros(shape, bool)
    solid[8:10, 4:7, 3:6] = True
    prob = workloads.channel_problem(shape=shape, steps=150, collision="trt", lattice=lattice, box_half_width=0,
                                     filter_radius_cells=2.0, solid=solid)
    prob["topology_map"]["projection_beta"] = 8.0
    prob["topology_map"]["projection_eta"] = 0.45
    rng = np.random.default_rng(21)
    fixed = rng.uniform(0.3, 1.0, size=shape)
    fixed[0] = fixed[nx - 1] = 1.0  # port cells must be fixed-design fluid (ports.rs:185-197)
    design = np.asarray(prob["design_region"]).copy()
    design[13:16, 2:5, 2:8] = False  # fixed override inside the channel
    prob["design_region"] = design
    prob["fixed_design"] = fixed
    return prob, solid, design


@pytest.mark.parametrize("lattice", ["D3Q19", "D3Q27"])
def test_conic_projection_channel_matches_oracle(gpu_lib, lattice):
    prob, solid, design = conic_channel(lattice)
    norm = normalize(prob)
    raw = workloads.uniform_design(norm.shape, 8)
    w = workloads.objective_weights()
    o = Oracle(norm)
    phi_r, alpha_r = o.design(raw)
    # the overrides are really exercised: solid cells map to 0, fixed cells
    # keep their value, editable cells see the projection
    assert np.all(phi_r.reshape(norm.shape)[solid] == 0.0)
    fixed_cells = ~design & ~solid
    np.testing.assert_array_equal(phi_r.reshape(norm.shape)[fixed_cells], np.asarray(prob["fixed_design"])[fixed_cells])
    f_r, d_r = o.history(alpha_r, norm.step_count)
    r_r = o.vector(phi_r, alpha_r, f_r)
    g_r, _, _, st = o.gradient(raw, w, mode="horizon", K=10)
    assert st == 0
    with LbmSolver(norm) as s:
        s.set_design(raw)
        phi, alpha = s.design()
        assert np.max(np.abs(phi.ravel() - phi_r)) < 1e-6
        assert rel_max(alpha, alpha_r) < 1e-5
        d = s.forward()
        assert d.admitted and d_r.admitted
        assert rel_max(s.populations(), f_r) < 1e-5
        r = s.responses()
        for k in (0, 3, 4, 5, 6, 7):
            assert abs(r[k] - r_r[k]) <= 1e-5 * abs(r_r[k]), (k, r[k], r_r[k])
        grad, _ = s.gradient(w, mode="horizon", checkpoint_every=10)
        assert rel_l2(grad, g_r) < 1e-4
        # the design-map transpose alone, on a random phi cotangent
        pb = np.random.default_rng(3).standard_normal(s.cells)
        assert rel_l2(s.design_vjp(pb), o.design_vjp(raw, pb)) < 1e-5
