"""Parity of the CUDA library (through its C-ABI) with the FP64 oracle.

Tolerances (FP32 arithmetic and storage unless stated):
  populations / velocity / density   max |gpu - ref| / max |ref| <= 1e-5
  responses                          relative 1e-5 (transverse mean velocities
                                     against 1e-5 of the axial one)
  one transposed step                relative L2 <= 1e-5
  design gradient                    relative L2 <= 1e-4
  FP16 / BF16 storage (vs FP64)      velocity 2e-3 / 2e-2, gradient relative
                                     L2 <= 1e-3 / 1e-2
"""
import numpy as np
import pytest

from implexity_b200 import LbmSolver, normalize, workloads
from oracle.oracle import Oracle

pytestmark = pytest.mark.gpu


def rel_l2(a, b):
    a, b = np.asarray(a, float).ravel(), np.asarray(b, float).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def rel_max(a, b):
    a, b = np.asarray(a, float).ravel(), np.asarray(b, float).ravel()
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def macroscopic(f, q, alpha, a_lat):
    """rho and the Brinkman-corrected velocity of populations f[cells, q]."""
    from oracle.oracle import lib  # noqa: F401  (keeps the oracle build fresh)

    if q == 19:
        c = np.array(
            [[0, 0, 0], [-1, -1, 0], [-1, 0, -1], [-1, 0, 0], [-1, 0, 1], [-1, 1, 0], [0, -1, -1], [0, -1, 0],
             [0, -1, 1], [0, 0, -1], [0, 0, 1], [0, 1, -1], [0, 1, 0], [0, 1, 1], [1, -1, 0], [1, 0, -1], [1, 0, 0],
             [1, 0, 1], [1, 1, 0]], float)
    else:
        c = np.array([[0, 0, 0]] + [[a, b, d] for a in (-1, 0, 1) for b in (-1, 0, 1) for d in (-1, 0, 1)
                                    if (a, b, d) != (0, 0, 0)], float)
    rho = f.sum(1)
    u = (f @ c / rho[:, None] + 0.5 * np.asarray(a_lat)) / (1 + 0.5 * alpha[:, None])
    return rho, u


CASES = [
    ("bgk", "D3Q19"),
    ("trt", "D3Q19"),
    ("mrt", "D3Q19"),
    ("trt", "D3Q27"),
    ("mrt", "D3Q27"),
]


def make(coll, lattice, shape=(16, 10, 8), steps=120, storage="float32", seed=1, **kw):
    prob = workloads.channel_problem(
        shape=shape, steps=steps, collision=coll, lattice=lattice, storage=storage,
        mrt_bulk_rate=1.2 if coll == "mrt" else None, **kw,
    )
    norm = normalize(prob)
    raw = workloads.uniform_design(norm.shape, seed)
    return prob, norm, raw


@pytest.mark.parametrize("coll,lattice", CASES)
def test_forward_matches_oracle(gpu_lib, coll, lattice):
    prob, norm, raw = make(coll, lattice)
    o = Oracle(norm)
    phi_ref, alpha_ref = o.design(raw)
    f_ref, d_ref = o.history(alpha_ref, norm.step_count)
    with LbmSolver(prob) as s:
        s.set_design(raw)
        phi, alpha = s.design()
        assert rel_max(phi, phi_ref) < 1e-6
        assert rel_max(alpha, alpha_ref) < 1e-5
        d = s.forward()
        f = s.populations()
        assert rel_max(f, f_ref) < 1e-5
        rho, u = macroscopic(f, s.q, alpha_ref, o.acceleration_lattice)
        rho_r, u_r = macroscopic(f_ref, s.q, alpha_ref, o.acceleration_lattice)
        assert rel_max(u, u_r) < 1e-5
        assert np.max(np.abs(rho - rho_r)) < 1e-5
        assert d.admitted and d_ref.admitted
        assert abs(d.maximum_mach - d_ref.maximum_mach) < 1e-5 * d_ref.maximum_mach
        assert abs(d.relative_mass_drift - d_ref.relative_mass_drift) < 1e-7
        r = s.responses()
        r_ref = o.vector(phi_ref, alpha_ref, f_ref)
        for k in (0, 3, 4, 5, 6, 7):
            assert abs(r[k] - r_ref[k]) <= 1e-5 * abs(r_ref[k]), (k, r[k], r_ref[k])
        for k in (1, 2):
            assert abs(r[k] - r_ref[k]) <= 1e-5 * abs(r_ref[0])


@pytest.mark.parametrize("lattice", ["D3Q19", "D3Q27"])
def test_periodic_solid_body_force(gpu_lib, lattice):
    """Periodic x/z, closed y walls, solid obstacles next to periodic faces,
    body force and no ports: the wrap and solid-neighbour bounce-back paths."""
    shape = (12, 9, 8)
    solid = np.zeros(shape, bool)
    solid[0, 3:5, 0:2] = True
    solid[6:8, 4, 3:6] = True
    prob = workloads.channel_problem(shape=shape, steps=150, collision="trt", lattice=lattice, ports=False, solid=solid)
    prob["periodic_axes"] = [True, False, True]
    prob["acceleration_m_s2"] = [2e-5, 0.0, 1e-6]
    prob["design_region"] = ~solid
    prob["design_region"][:, 0, :] = False
    norm = normalize(prob)
    raw = workloads.uniform_design(shape, 4)
    o = Oracle(norm)
    phi_r, alpha_r = o.design(raw)
    f_r, d_r = o.history(alpha_r, norm.step_count)
    with LbmSolver(prob) as s:
        s.set_design(raw)
        d = s.forward()
        f = s.populations()
        assert rel_max(f, f_r) < 1e-5
        assert d.admitted == bool(d_r.admitted)
        assert abs(d.relative_mass_drift - d_r.relative_mass_drift) < 1e-7


@pytest.mark.parametrize("storage", ["float32", "float16"])
def test_unaligned_grid_matches_oracle(gpu_lib, storage):
    """A grid whose plane stride and strides are not multiples of the 16-byte
    vector: the stepping kernels take their run offsets from the table and the
    last partial tile of every plane stores directly."""
    prob, norm, raw = make("trt", "D3Q19", shape=(11, 7, 5), steps=80, storage=storage)
    o = Oracle(norm)
    _, alpha = o.design(raw)
    f_ref, _ = o.history(alpha, norm.step_count)
    w = workloads.objective_weights()
    g_ref, _, _, st = o.gradient(raw, w, mode="horizon", K=20)
    assert st == 0
    with LbmSolver(prob) as s:
        s.set_design(raw)
        s.forward()
        f = s.populations()
        g, _ = s.gradient(w, mode="horizon", checkpoint_every=20,
                          lambda_storage=storage)
    tol_f, tol_g = (1e-5, 1e-4) if storage == "float32" else (2e-3, 2e-3)
    assert rel_max(f, f_ref) < tol_f
    assert rel_l2(g, g_ref) < tol_g, rel_l2(g, g_ref)


@pytest.mark.parametrize("coll,lattice", CASES)
def test_step_vjp_matches_oracle(gpu_lib, coll, lattice):
    prob, norm, raw = make(coll, lattice, steps=40)
    o = Oracle(norm)
    _, alpha = o.design(raw)
    state, _ = o.history(alpha, 40)
    rng = np.random.default_rng(7)
    lam_next = rng.standard_normal(state.shape)
    lam_ref, ab_ref = o.interval_vjp(state, alpha, lam_next)
    with LbmSolver(prob) as s:
        s.set_design(raw)
        lam, ab = s.step_vjp(state, lam_next)
    assert rel_l2(lam, lam_ref) < 1e-5
    assert rel_l2(ab, ab_ref) < 1e-5


@pytest.mark.parametrize("coll,lattice", [("bgk", "D3Q19"), ("trt", "D3Q19"), ("mrt", "D3Q27")])
@pytest.mark.parametrize("response", [0, 3, 4, 5, 6, 7])
def test_horizon_gradient_matches_oracle(gpu_lib, coll, lattice, response):
    prob, norm, raw = make(coll, lattice, steps=60)
    w = np.zeros(8)
    w[response] = 1.0
    o = Oracle(norm)
    g_ref, r_ref, _, st = o.gradient(raw, w, mode="horizon", K=13)
    assert st == 0
    with LbmSolver(prob) as s:
        s.set_design(raw)
        g, rep = s.gradient(w, mode="horizon", checkpoint_every=13)
    # the fluid volume does not depend on the populations: no adjoint steps needed
    assert rep.iterations == (0 if response == 5 else 60)
    assert rel_l2(g, g_ref) < 1e-4, rel_l2(g, g_ref)


def test_steady_gradient_matches_oracle(gpu_lib):
    prob, norm, raw = make("trt", "D3Q19", steps=1500)
    w = workloads.objective_weights()
    o = Oracle(norm)
    g_ref, r_ref, rep_ref, st = o.gradient(raw, w, mode="steady", tol=1e-12)
    assert st == 0
    with LbmSolver(prob) as s:
        s.set_design(raw)
        s.forward()
        r = s.responses()
        g, rep = s.gradient(w, mode="steady", tolerance=1e-8)
    assert rep.converged
    assert abs(np.dot(w, r) - np.dot(w, r_ref)) <= 1e-6 * abs(np.dot(w, r_ref)) + 1e-12
    assert rel_l2(g, g_ref) < 1e-4, rel_l2(g, g_ref)


def _sixteen_bit_against_oracle(storage, u_tol, g_tol):
    """16-bit storage of (f - w)/w against the FP64 oracle: velocity of the
    final state (max norm) and the steady gradient (relative L2)."""
    prob, norm, raw = make("trt", "D3Q19", steps=600, storage=storage)
    w = workloads.objective_weights()
    o = Oracle(norm)
    _, alpha = o.design(raw)
    f_ref, _ = o.history(alpha, norm.step_count)
    g_ref, _, _, st = o.gradient(raw, w, mode="steady", tol=1e-12)
    assert st == 0
    with LbmSolver(prob) as s:
        s.set_design(raw)
        s.forward()
        f = s.populations()
        g, rep = s.gradient(w, mode="steady", tolerance=1e-8, lambda_storage=storage)
    assert rep.converged
    _, u = macroscopic(f, 19, alpha, o.acceleration_lattice)
    _, u_ref = macroscopic(f_ref, 19, alpha, o.acceleration_lattice)
    assert rel_max(u, u_ref) < u_tol, rel_max(u, u_ref)
    assert rel_l2(g, g_ref) < g_tol, rel_l2(g, g_ref)


def test_fp16_storage_against_fp64_oracle(gpu_lib):
    """FP16 storage (10 mantissa bits): velocity 2e-3, gradient 1e-3."""
    _sixteen_bit_against_oracle("float16", 2e-3, 1e-3)


def solid_channel(lattice, storage="float32", steps=60, periodic=(False, False, False)):
    """Channel with solid obstacles touching the y/z walls, the inlet face and
    each other: blocked links of every kind (walls, solids, edges, corners)."""
    shape = (14, 9, 8)
    solid = np.zeros(shape, bool)
    solid[4:6, 0:3, 0:2] = True      # in the y=0 / z=0 corner
    solid[8, 4, 3:8] = True          # a plate reaching the z = nz-1 wall
    solid[10:12, 6:9, 5] = True      # touching the y = ny-1 wall
    solid[1, 2, 2] = True            # next to the inlet plane
    prob = workloads.channel_problem(shape=shape, steps=steps, collision="trt", lattice=lattice, storage=storage,
                                     solid=solid)
    prob["periodic_axes"] = list(periodic)
    norm = normalize(prob)
    return prob, norm, workloads.uniform_design(shape, 3)


@pytest.mark.parametrize("lattice", ["D3Q19", "D3Q27"])
def test_solid_channel_horizon_gradient_matches_oracle(gpu_lib, lattice):
    """Transposed steps over walls and solids: every blocked link of the
    transposed pull reads the cell's own opposite slot."""
    prob, norm, raw = solid_channel(lattice)
    w = workloads.objective_weights()
    o = Oracle(norm)
    g_ref, _, _, st = o.gradient(raw, w, mode="horizon", K=11)
    assert st == 0
    with LbmSolver(prob) as s:
        s.set_design(raw)
        g, rep = s.gradient(w, mode="horizon", checkpoint_every=11)
    assert rep.iterations == 60
    assert rel_l2(g, g_ref) < 1e-4, rel_l2(g, g_ref)


@pytest.mark.parametrize("lattice", ["D3Q19", "D3Q27"])
def test_solid_channel_step_vjp_matches_oracle(gpu_lib, lattice):
    prob, norm, raw = solid_channel(lattice, steps=30)
    o = Oracle(norm)
    _, alpha = o.design(raw)
    state, _ = o.history(alpha, 30)
    lam_next = np.random.default_rng(11).standard_normal(state.shape)
    lam_ref, ab_ref = o.interval_vjp(state, alpha, lam_next)
    with LbmSolver(prob) as s:
        s.set_design(raw)
        lam, ab = s.step_vjp(state, lam_next)
    fluid = ~np.asarray(norm.solid_mask, bool).reshape(-1)
    assert rel_l2(lam[fluid], lam_ref[fluid]) < 1e-5
    assert rel_l2(ab, ab_ref) < 1e-5


def test_solid_channel_steady_gradient_matches_oracle(gpu_lib):
    prob, norm, raw = solid_channel("D3Q19", steps=1200)
    w = workloads.objective_weights()
    o = Oracle(norm)
    g_ref, _, _, st = o.gradient(raw, w, mode="steady", tol=1e-12)
    assert st == 0
    with LbmSolver(prob) as s:
        s.set_design(raw)
        s.forward()
        g, rep = s.gradient(w, mode="steady", tolerance=1e-8)
    assert rep.converged
    assert rel_l2(g, g_ref) < 1e-4, rel_l2(g, g_ref)


def test_periodic_solid_horizon_gradient_matches_oracle(gpu_lib):
    """Transposed steps across periodic faces (the wrap path) next to solids."""
    shape = (12, 9, 8)
    solid = np.zeros(shape, bool)
    solid[0, 3:5, 0:2] = True
    solid[6:8, 4, 3:6] = True
    prob = workloads.channel_problem(shape=shape, steps=50, collision="trt", ports=False, solid=solid)
    prob["periodic_axes"] = [True, False, True]
    prob["acceleration_m_s2"] = [2e-5, 0.0, 1e-6]
    prob["design_region"] = ~solid
    norm = normalize(prob)
    raw = workloads.uniform_design(shape, 4)
    w = np.zeros(8)
    w[7] = 1.0
    o = Oracle(norm)
    g_ref, _, _, st = o.gradient(raw, w, mode="horizon", K=9)
    assert st == 0
    with LbmSolver(prob) as s:
        s.set_design(raw)
        g, _ = s.gradient(w, mode="horizon", checkpoint_every=9)
    assert rel_l2(g, g_ref) < 1e-4, rel_l2(g, g_ref)


def test_bounded_wait_runs_out_and_the_context_stays_usable(gpu_lib):
    """A wait that nothing completes gives up after its limit, reports it
    through the error flag and returns; the next solve runs normally."""
    import ctypes as C

    timed_out, waited = C.c_int32(0), C.c_double(0.0)
    assert gpu_lib.lbm_probe_bounded_wait(50_000_000, C.byref(timed_out), C.byref(waited)) == 0
    assert timed_out.value == 1
    assert 50.0 <= waited.value < 2000.0, waited.value
    prob, norm, raw = make("trt", "D3Q19", steps=20)
    with LbmSolver(prob) as s:
        s.set_design(raw)
        d = s.forward()
        assert d.admitted


@pytest.mark.parametrize("lattice,coll,storage", [("D3Q19", "trt", "float32"), ("D3Q27", "trt", "float32"),
                                                  ("D3Q19", "bgk", "float32"), ("D3Q19", "trt", "float16")])
def test_wall_loads_match_oracle(gpu_lib, lattice, coll, storage):
    """Momentum-exchange loads of the last interval (wall_exchange.rs): every
    blocked link of walls and solids except the port faces, from the state
    before the last step collided with Guo-BGK."""
    shape = (14, 9, 8)
    solid = np.zeros(shape, bool)
    solid[4:6, 0:3, 0:2] = True
    solid[8, 4, 3:8] = True
    solid[1, 2, 2] = True
    steps = 40
    prob = workloads.channel_problem(shape=shape, steps=steps, collision=coll, lattice=lattice, storage=storage,
                                     solid=solid)
    prob["origin_m"] = [0.01, -0.02, 0.003]
    norm = normalize(prob)
    raw = workloads.uniform_design(shape, 3)
    o = Oracle(norm)
    _, alpha = o.design(raw)
    before, _ = o.history(alpha, steps - 1)
    datum = 12.5
    f_ref = o.wall_loads(before, alpha, datum)
    with LbmSolver(prob) as s:
        s.set_design(raw)
        s.forward()
        loads = s.wall_loads(datum)
    pos, force = loads["wall_link_positions_m"], loads["wall_link_gauge_force_N"]
    assert force.shape == f_ref.shape and len(force) > 0
    tol = 1e-5 if storage == "float32" else 2e-3
    assert np.max(np.abs(force - f_ref)) <= tol * np.max(np.abs(f_ref))
    # link midpoints: origin + (ijk + 1/2 - c_q / 2) dx, links in (cell, q) order
    assert np.all(np.isfinite(pos))
    dx = norm.spacing_m
    ijk = np.rint((pos - np.array(prob["origin_m"])) / dx - 0.5)
    assert np.all(np.abs((pos - np.array(prob["origin_m"])) / dx - 0.5 - ijk) <= 0.5 + 1e-9)


@pytest.mark.parametrize("lattice", ["D3Q19", "D3Q27"])
def test_mrt_with_even_rate_matches_oracle(gpu_lib, lattice):
    """MRT with a bulk and an even-high rate (two rank-one corrections: the
    general branch; a bulk rate alone takes the compile-time folded one)."""
    prob = workloads.channel_problem(shape=(16, 10, 8), steps=60, collision="mrt", lattice=lattice, mrt_bulk_rate=1.2)
    prob["solver_options"]["collision"]["even_rate"] = 1.1
    norm = normalize(prob)
    raw = workloads.uniform_design(norm.shape, 1)
    o = Oracle(norm)
    _, alpha = o.design(raw)
    f_ref, _ = o.history(alpha, 60)
    w = workloads.objective_weights()
    g_ref, _, _, st = o.gradient(raw, w, mode="horizon", K=12)
    assert st == 0
    with LbmSolver(norm) as s:
        s.set_design(raw)
        s.forward()
        f = s.populations()
        g, _ = s.gradient(w, mode="horizon", checkpoint_every=12)
    assert rel_max(f, f_ref) < 1e-5
    assert rel_l2(g, g_ref) < 1e-4, rel_l2(g, g_ref)


def test_bf16_storage_against_fp64_oracle(gpu_lib):
    """BF16 storage (7 mantissa bits): velocity 2e-2, gradient 1e-2."""
    _sixteen_bit_against_oracle("bfloat16", 2e-2, 1e-2)


def test_nonfinite_population_in_a_solid_cell_is_refused(gpu_lib):
    """admit (solver.rs:714-719) checks finiteness over every cell, solid ones
    included, and the minimum over fluid cells: a NaN loaded into a solid cell
    refuses the trajectory; a clean reload is admitted again."""
    from implexity_b200 import ContractError

    shape = (12, 9, 8)
    solid = np.zeros(shape, bool)
    solid[5:7, 3:5, 3:5] = True
    prob = workloads.channel_problem(shape=shape, steps=20, collision="trt", solid=solid)
    raw = workloads.uniform_design(shape, 2)
    with LbmSolver(prob) as s:
        s.set_design(raw)
        s.forward()
        f = s.populations()
        bad = f.copy()
        bad[int(np.flatnonzero(solid.ravel())[0]), 4] = np.nan
        s.set_populations(bad)
        with pytest.raises(ContractError, match="nonpositive or nonfinite"):
            s.advance(3)
        assert s.last_diag.nonfinite
        s.set_populations(f)
        assert s.advance(3).admitted
