"""The nonlinear port reconstructions: the two that rebuild a port cell from
its inward neighbour, ports.rs's neighbor_non_equilibrium (:484-497) and the
moving engine's non-equilibrium extrapolation (moving/boundary.rs:445-506,
port_populations and its VJP), and ports.rs's regularized_known_stress
(:409-482), which rebuilds every population from the cell's own legacy
target and a stress fitted to its known populations.

CPU: the oracle's transposed interval with these ports against FP64 central
differences of one interval (directional, on the state).
GPU (through the C-ABI, against the oracle): trajectory (1e-5), responses
(1e-5), one transposed step (1e-5 relative L2), horizon and steady gradients
(1e-4 relative L2).
"""
import numpy as np
import pytest

from implexity_b200 import LbmSolver, normalize, workloads
from oracle.oracle import Oracle


def _rel_l2(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def nee_channel(inlet, outlet, lattice="D3Q19", shape=(14, 8, 7), steps=120, collision="trt", storage="float32"):
    """The channel with the inlet / outlet reconstructions given (a solid
    block in the middle)."""
    solid = np.zeros(shape, bool)
    solid[6:8, 3:5, 2:4] = True
    prob = workloads.channel_problem(shape=shape, steps=steps, collision=collision, lattice=lattice, solid=solid,
                                     storage=storage, u_in=0.04)
    prob["ports"][0]["reconstruction"] = inlet
    prob["ports"][1]["reconstruction"] = outlet
    # the extrapolations read protected, fixed-design inward planes (ports.rs:202-219)
    design = np.asarray(prob["design_region"], bool).copy()
    design[1] = design[-2] = False
    prob["design_region"] = design
    return prob


CASES = [
    ("legacy_moment", "neighbor_non_equilibrium", "D3Q19"),
    ("non_equilibrium_extrapolation", "non_equilibrium_extrapolation", "D3Q19"),
    ("non_equilibrium_extrapolation", "neighbor_non_equilibrium", "D3Q27"),
    ("regularized_known_stress", "regularized_known_stress", "D3Q19"),
    ("regularized_known_stress", "neighbor_non_equilibrium", "D3Q27"),
]


@pytest.mark.parametrize("inlet,outlet,lattice", CASES)
def test_oracle_transposed_interval_matches_central_differences(inlet, outlet, lattice):
    norm = normalize(nee_channel(inlet, outlet, lattice, steps=10))
    o = Oracle(norm)
    _, alpha = o.design(workloads.uniform_design(norm.shape, 2))
    f, d = o.history(alpha, 10)
    assert d.admitted
    rng = np.random.default_rng(5)
    after_bar = rng.standard_normal(f.shape)
    fb, _ = o.interval_vjp(f, alpha, after_bar)
    solid = np.asarray(norm.solid_mask, bool).reshape(-1)
    dirn = rng.standard_normal(f.shape) * 1e-3
    dirn[solid] = 0.0  # solid cells carry their populations unchanged
    h = 1e-3  # state perturbations of ~1e-6: far from FP64 rounding, truncation ~1e-12

    def J(state):
        out, _ = o.interval(state, alpha)
        return float(np.sum(after_bar * out))

    fd = (J(f + h * dirn) - J(f - h * dirn)) / (2 * h)
    assert abs(fd - float(np.sum(fb * dirn))) <= 1e-7 * abs(fd)


def test_extrapolations_need_zero_acceleration_and_a_pressure_port():
    from implexity_b200 import ContractError

    prob = nee_channel("neighbor_non_equilibrium", "legacy_moment")
    with pytest.raises(ContractError, match="pressure port and zero acceleration"):
        _create(prob)
    prob = nee_channel("legacy_moment", "non_equilibrium_extrapolation")
    prob["acceleration_m_s2"] = [1e-6, 0.0, 0.0]
    with pytest.raises(ContractError, match="zero acceleration"):
        _create(prob)
    prob = nee_channel("regularized_known_stress", "legacy_moment")
    prob["acceleration_m_s2"] = [0.0, 1e-6, 0.0]
    with pytest.raises(ContractError, match="regularized_known_stress ports require zero acceleration"):
        _create(prob)
    # the inward plane must be protected fluid
    prob = nee_channel("legacy_moment", "neighbor_non_equilibrium")
    design = np.asarray(prob["design_region"], bool).copy()
    design[-2, 3, 3] = True
    prob["design_region"] = design
    with pytest.raises(ContractError, match="protected, unobstructed, fixed-design inward fluid cells"):
        _create(prob)


def test_regularized_port_keeps_the_legacy_density_and_velocity():
    """The rebuilt cell carries the legacy target's density and momentum: the
    stress basis has neither (the fact the transposed port relies on)."""
    norm = normalize(nee_channel("regularized_known_stress", "regularized_known_stress", steps=10))
    o = Oracle(norm)
    _, alpha = o.design(workloads.uniform_design(norm.shape, 2))
    f, _ = o.history(alpha, 10)
    norm_l = normalize(nee_channel("legacy_moment", "legacy_moment", steps=10))
    ol = Oracle(norm_l)
    rng = np.random.default_rng(3)
    cells = np.flatnonzero(np.asarray(norm.ports[0]["mask"]).reshape(-1))
    for x in rng.choice(cells, 4, replace=False):
        src = f[x] + 1e-3 * rng.standard_normal(f.shape[1])
        reg = o.port_apply(0, src)
        leg = ol.port_apply(0, src)
        c = np.array([[0, 0, 0], [-1, -1, 0], [-1, 0, -1], [-1, 0, 0], [-1, 0, 1], [-1, 1, 0], [0, -1, -1],
                      [0, -1, 0], [0, -1, 1], [0, 0, -1], [0, 0, 1], [0, 1, -1], [0, 1, 0], [0, 1, 1], [1, -1, 0],
                      [1, 0, -1], [1, 0, 0], [1, 0, 1], [1, 1, 0]], float)
        np.testing.assert_allclose(reg.sum(), leg.sum(), rtol=1e-13)
        np.testing.assert_allclose(reg @ c, leg @ c, atol=1e-14)
        assert np.max(np.abs(reg - leg)) > 1e-6  # the known populations are rebuilt too


def test_slab_handles_take_legacy_ports_only():
    import ctypes as C

    from implexity_b200 import ContractError, _abi
    from implexity_b200.solver import _raise

    norm = normalize(nee_channel("legacy_moment", "neighbor_non_equilibrium"))
    lib = _abi.load()
    cp = norm.to_c()
    h = C.c_void_p()
    st = lib.lbm_create_slab(C.byref(cp), 0, norm.shape[0] // 2, 1, C.byref(h))
    assert st != _abi.LBM_OK
    with pytest.raises(ContractError, match="legacy_moment ports only"):
        _raise(st, lib.lbm_last_error(None).decode())


def _create(prob):
    """lbm_create's validation only (no device needed when it refuses)."""
    import ctypes as C

    from implexity_b200 import _abi
    from implexity_b200.solver import _raise

    norm = normalize(prob)
    lib = _abi.load()
    cp = norm.to_c()
    h = C.c_void_p()
    st = lib.lbm_create(C.byref(cp), C.byref(h))
    if st != _abi.LBM_OK:
        _raise(st, lib.lbm_last_error(None).decode())
    lib.lbm_destroy(h)


@pytest.mark.gpu
@pytest.mark.parametrize("inlet,outlet,lattice", CASES)
def test_extrapolating_ports_match_oracle(gpu_lib, inlet, outlet, lattice):
    norm = normalize(nee_channel(inlet, outlet, lattice))
    raw = workloads.uniform_design(norm.shape, 4)
    w = workloads.objective_weights()
    o = Oracle(norm)
    phi_r, alpha_r = o.design(raw)
    f_r, d_r = o.history(alpha_r, norm.step_count)
    r_r = o.vector(phi_r, alpha_r, f_r)
    g_h, _, _, st = o.gradient(raw, w, mode="horizon", K=20)
    assert st == 0
    lam_next = np.random.default_rng(8).standard_normal(f_r.shape)
    fb_r, ab_r = o.interval_vjp(f_r, alpha_r, lam_next)
    with LbmSolver(norm) as s:
        s.set_design(raw)
        d = s.forward()
        assert d.admitted and d_r.admitted
        f = s.populations()
        assert float(np.max(np.abs(f - f_r)) / np.max(np.abs(f_r))) < 1e-5
        assert abs(d.relative_mass_drift - d_r.relative_mass_drift) < 1e-7
        r = s.responses()
        for k in (0, 3, 4, 6, 7):
            assert abs(r[k] - r_r[k]) <= 1e-5 * abs(r_r[k]), (k, r[k], r_r[k])
        g, _ = s.gradient(w, mode="horizon", checkpoint_every=20)
        assert _rel_l2(g, g_h) < 1e-4, _rel_l2(g, g_h)
        fb, ab = s.step_vjp(f_r, lam_next)
    fluid = ~np.asarray(norm.solid_mask, bool).reshape(-1)
    assert _rel_l2(fb[fluid], fb_r[fluid]) < 1e-5
    assert _rel_l2(ab, ab_r) < 1e-5


@pytest.mark.gpu
def test_extrapolating_ports_steady_gradient_matches_oracle(gpu_lib):
    norm = normalize(nee_channel("non_equilibrium_extrapolation", "neighbor_non_equilibrium", steps=1500))
    raw = workloads.uniform_design(norm.shape, 9)
    w = workloads.objective_weights()
    g_ref, _, _, st = Oracle(norm).gradient(raw, w, mode="steady", tol=1e-12)
    assert st == 0
    with LbmSolver(norm) as s:
        s.set_design(raw)
        s.forward()
        g, rep = s.gradient(w, mode="steady", tolerance=1e-10)
    assert rep.converged
    assert _rel_l2(g, g_ref) < 1e-4, _rel_l2(g, g_ref)


@pytest.mark.gpu
@pytest.mark.parametrize("inlet,outlet", [("non_equilibrium_extrapolation", "neighbor_non_equilibrium"),
                                          ("regularized_known_stress", "regularized_known_stress")])
def test_nonlinear_ports_with_16_bit_storage(gpu_lib, inlet, outlet):
    """The 16-bit stepping path ((f - w)/w storage units) through the same
    ports, against the FP64 oracle at the 16-bit bars: velocity 2e-3 of its
    largest value, horizon gradient 1e-3 relative L2."""
    norm = normalize(nee_channel(inlet, outlet, storage="float16"))
    raw = workloads.uniform_design(norm.shape, 4)
    w = workloads.objective_weights()
    o = Oracle(norm)
    phi_r, alpha_r = o.design(raw)
    f_r, d_r = o.history(alpha_r, norm.step_count)
    g_h, _, _, st = o.gradient(raw, w, mode="horizon", K=20)
    assert st == 0
    from test_gpu_parity import macroscopic

    with LbmSolver(norm) as s:
        s.set_design(raw)
        d = s.forward()
        assert d.admitted
        f = s.populations()
        g, _ = s.gradient(w, mode="horizon", checkpoint_every=20)
    fluid = ~np.asarray(norm.solid_mask, bool).reshape(-1)
    a = np.asarray(o.acceleration_lattice)
    _, u = macroscopic(f[fluid], o.q, alpha_r[fluid], a)
    _, u_r = macroscopic(f_r[fluid], o.q, alpha_r[fluid], a)
    assert float(np.max(np.abs(u - u_r)) / np.max(np.abs(u_r))) < 2e-3
    assert _rel_l2(g, g_h) < 1e-3, _rel_l2(g, g_h)
