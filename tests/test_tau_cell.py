"""Per-cell relaxation times (Tau::PerCell, solver.rs:171-187) of the BGK
collision, as the reference's thermal provider steps with them.

CPU: the oracle's tau cotangent (collide_cell_vjp's tau_bar, solver.rs:214-285)
against FP64 central differences of one interval.
GPU (through the C-ABI, against the oracle with the same random tau field):
the trajectory and responses (1e-5), the horizon gradient (1e-4 relative L2),
and one step's VJP with its tau cotangent (1e-5 relative L2).
"""
import numpy as np
import pytest

from implexity_b200 import ContractError, LbmSolver, normalize, workloads
from oracle.oracle import Oracle


def _rel_l2(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def _problem(shape=(14, 9, 8), steps=80, collision="bgk", solid=True):
    mask = None
    if solid:
        mask = np.zeros(shape, bool)
        mask[6:8, 3:5, 2:5] = True
    return workloads.channel_problem(shape=shape, steps=steps, collision=collision, solid=mask)


def _tau_field(shape, seed=4):
    return np.random.default_rng(seed).uniform(0.6, 1.2, size=shape)


def test_oracle_tau_cotangent_matches_central_differences():
    norm = normalize(_problem(shape=(8, 6, 6), steps=10))
    o = Oracle(norm)
    raw = workloads.uniform_design(norm.shape, 3)
    _, alpha = o.design(raw)
    tau = _tau_field(norm.shape).ravel()
    o.set_tau(tau)
    f, _ = o.history(alpha, 10)
    rng = np.random.default_rng(9)
    after_bar = rng.standard_normal(f.shape)
    _, _, tau_bar = o.interval_vjp_tau(f, alpha, after_bar)
    solid = np.asarray(norm.solid_mask, bool).ravel()
    assert np.all(tau_bar[solid] == 0.0)
    d = rng.standard_normal(tau.size) * 0.05
    h = 1e-5

    def J(t):
        o.set_tau(t)
        out, _ = o.interval(f, alpha)
        return float(np.sum(after_bar * out))

    fd = (J(tau + h * d) - J(tau - h * d)) / (2 * h)
    assert abs(fd - float(np.dot(tau_bar, d))) <= 1e-7 * abs(fd)
    # a per-cell field of one value is the uniform tau
    o.set_tau(np.full(tau.size, norm.tau))
    a1, _ = o.interval(f, alpha)
    o.set_tau(None)
    a2, _ = o.interval(f, alpha)
    np.testing.assert_allclose(a1, a2, rtol=0, atol=1e-15)


@pytest.mark.gpu
def test_per_cell_tau_forward_and_gradient_match_oracle(gpu_lib):
    norm = normalize(_problem())
    raw = workloads.uniform_design(norm.shape, 5)
    tau = _tau_field(norm.shape)
    w = workloads.objective_weights()
    o = Oracle(norm)
    o.set_tau(tau)
    phi_r, alpha_r = o.design(raw)
    f_r, d_r = o.history(alpha_r, norm.step_count)
    r_r = o.vector(phi_r, alpha_r, f_r)
    g_r, _, _, st = o.gradient(raw, w, mode="horizon", K=20)
    assert st == 0
    with LbmSolver(norm) as s:
        s.set_tau(tau)
        s.set_design(raw)
        d = s.forward()
        assert d.admitted and d_r.admitted
        f = s.populations()
        assert float(np.max(np.abs(f - f_r)) / np.max(np.abs(f_r))) < 1e-5
        r = s.responses()
        for k in (0, 3, 4, 6):
            assert abs(r[k] - r_r[k]) <= 1e-5 * abs(r_r[k]), (k, r[k], r_r[k])
        g, _ = s.gradient(w, mode="horizon", checkpoint_every=20)
        assert _rel_l2(g, g_r) < 1e-4, _rel_l2(g, g_r)
        # the uniform tau again: the field is dropped
        s.set_tau(None)
        s.forward()
        o2 = Oracle(norm)
        f_u, _ = o2.history(alpha_r, norm.step_count)
        assert float(np.max(np.abs(s.populations() - f_u)) / np.max(np.abs(f_u))) < 1e-5


@pytest.mark.gpu
def test_step_vjp_with_tau_cotangent_matches_oracle(gpu_lib):
    norm = normalize(_problem())
    raw = workloads.uniform_design(norm.shape, 6)
    tau = _tau_field(norm.shape, seed=7)
    o = Oracle(norm)
    o.set_tau(tau)
    _, alpha = o.design(raw)
    f, _ = o.history(alpha, 30)
    lam_next = np.random.default_rng(2).standard_normal(f.shape)
    fb_r, ab_r, tb_r = o.interval_vjp_tau(f, alpha, lam_next)
    with LbmSolver(norm) as s:
        s.set_tau(tau)
        s.set_design(raw)
        fb, ab, tb = s.step_vjp_tau(f, lam_next)
    # solid cells carry their state unchanged; the step's cotangent of their
    # slots is compared through the fluid cells that read them
    fluid = ~np.asarray(norm.solid_mask, bool).reshape(-1)
    assert _rel_l2(fb[fluid], fb_r[fluid]) < 1e-5
    assert _rel_l2(ab, ab_r) < 1e-5
    assert _rel_l2(tb, tb_r) < 1e-5, _rel_l2(tb, tb_r)


@pytest.mark.gpu
def test_per_cell_tau_contract(gpu_lib):
    with LbmSolver(normalize(_problem(collision="trt"))) as s:
        with pytest.raises(ContractError, match="BGK"):
            s.set_tau(_tau_field(s.shape))
    with LbmSolver(normalize(_problem())) as s:
        bad = _tau_field(s.shape)
        bad[0, 0, 0] = 0.5
        with pytest.raises(ContractError, match="greater than 0.5"):
            s.set_tau(bad)
