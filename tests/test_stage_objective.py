"""Pulsatile ports and the time-averaged (stage) objective.

The inlet follows the moving engine's port signal (moving/boundary.rs:98-126;
value at time t, moving/field.rs:1002-1013); the objective is the mean of the
weighted responses over the states 1..T, so every state seeds the adjoint.
No reference test covers either, so the oracle's stage gradient is pinned by
FP64 central differences (CPU), and the GPU is compared with the oracle:
populations 1e-5 relative, time-averaged responses 1e-5, gradient 1e-4
relative L2 (FP32 storage).
"""
import numpy as np
import pytest

from implexity_b200 import LbmSolver, normalize, workloads
from implexity_b200.problem import ContractError
from oracle.oracle import Oracle


def rel_l2(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def rel_max(a, b):
    a, b = np.ravel(a), np.ravel(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def small(lattice="D3Q19", steps=40, shape=(10, 7, 6)):
    prob = workloads.pulsatile_problem(shape=shape, steps=steps, lattice=lattice, u_mean=0.04, amp_frac=0.5,
                                       period_steps=16, ramp_steps=6, box_half_width=1)
    return prob, normalize(prob), workloads.uniform_design(shape, 2)


# ---------------------------------------------------------------- CPU (oracle)
@pytest.mark.parametrize("lattice", ["D3Q19", "D3Q27"])
def test_oracle_stage_gradient_matches_central_differences(lattice):
    prob, norm, raw = small(lattice, steps=24, shape=(8, 6, 5))
    o = Oracle(norm)
    w = workloads.objective_weights()
    g, r, _, st = o.gradient(raw, w, mode="time_average", K=7)
    assert st == 0
    editable = np.asarray(norm.design_region, bool).reshape(norm.shape)
    rng = np.random.default_rng(5)
    h = 1e-6
    for _ in range(2):
        d = np.where(editable & (raw > 2 * h) & (raw < 1 - 2 * h), rng.standard_normal(norm.shape), 0.0)
        jp = np.dot(w, o.gradient(raw + h * d, w, mode="time_average", K=7)[1])
        jm = np.dot(w, o.gradient(raw - h * d, w, mode="time_average", K=7)[1])
        fd = (jp - jm) / (2 * h)
        ad = float(np.sum(g * d.ravel()))
        assert abs(fd - ad) <= 1e-6 * abs(ad), (fd, ad)


def test_oracle_stage_objective_of_one_step_is_the_final_objective():
    prob = workloads.channel_problem(shape=(8, 6, 5), steps=1, collision="trt")
    prob["solver_options"]["time_average"] = True
    norm = normalize(prob)
    raw = workloads.uniform_design((8, 6, 5), 1)
    o = Oracle(norm)
    w = workloads.objective_weights()
    g0, r0, _, _ = o.gradient(raw, w, mode="horizon")
    g2, r2, _, _ = o.gradient(raw, w, mode="time_average")
    np.testing.assert_allclose(r2, r0, rtol=1e-14, atol=0)
    np.testing.assert_allclose(g2, g0, rtol=1e-12, atol=1e-30)


def test_signal_contract_messages():
    prob, _, _ = small()
    bad = dict(prob)
    bad["ports"] = [dict(p) for p in prob["ports"]]
    bad["ports"][0]["frequency_hz"] = -1.0
    with pytest.raises(ContractError, match="frequency_hz"):
        normalize(bad)
    bad["ports"][0]["frequency_hz"] = 1.0
    bad["ports"][0]["amplitude_Pa"] = 1.0  # a velocity port has no pressure amplitude
    with pytest.raises(ContractError, match="exact port fields"):
        normalize(bad)


# ---------------------------------------------------------------- GPU
@pytest.mark.gpu
@pytest.mark.parametrize("lattice", ["D3Q19", "D3Q27"])
def test_pulsatile_forward_and_time_average_match_oracle(gpu_lib, lattice):
    prob, norm, raw = small(lattice)
    o = Oracle(norm)
    _, alpha = o.design(raw)
    f_ref, _ = o.history(alpha, norm.step_count)
    w = workloads.objective_weights()
    _, r_ref, _, st = o.gradient(raw, w, mode="time_average", K=10)
    assert st == 0
    with LbmSolver(norm) as s:
        s.set_design(raw)
        s.forward()
        f = s.populations()
        avg = s.time_average()
    assert rel_max(f, f_ref) < 1e-5
    for k in (0, 3, 4, 5, 6, 7):
        assert abs(avg[k] - r_ref[k]) <= 1e-5 * abs(r_ref[k]), (k, avg[k], r_ref[k])


@pytest.mark.gpu
@pytest.mark.parametrize("lattice", ["D3Q19", "D3Q27"])
def test_time_averaged_gradient_matches_oracle(gpu_lib, lattice):
    prob, norm, raw = small(lattice)
    o = Oracle(norm)
    w = workloads.objective_weights()
    g_ref, _, _, st = o.gradient(raw, w, mode="time_average", K=10)
    assert st == 0
    with LbmSolver(norm) as s:
        s.set_design(raw)
        g, rep = s.gradient(w, mode="horizon", checkpoint_every=10, objective="time_average")
    assert rep.iterations == norm.step_count
    assert rel_l2(g, g_ref) < 1e-4, rel_l2(g, g_ref)


@pytest.mark.gpu
def test_time_average_requires_the_problem_option(gpu_lib):
    prob = workloads.channel_problem(shape=(10, 7, 6), steps=10, collision="trt")
    with LbmSolver(prob) as s:
        s.set_design(workloads.uniform_design((10, 7, 6), 0))
        s.forward()
        with pytest.raises(ContractError, match="time_average"):
            s.gradient(workloads.objective_weights(), objective="time_average")


@pytest.mark.gpu
def test_two_level_checkpoints_match_one_level(gpu_lib):
    """A record budget smaller than a segment's records splits each segment
    into spans (a second checkpoint level): same gradient, one more
    recomputed forward per segment."""
    prob, norm, raw = small("D3Q19", steps=40)
    w = workloads.objective_weights()
    rec_bytes = norm.cells * 10 * 4
    with LbmSolver(norm) as s:
        s.set_design(raw)
        g1, r1 = s.gradient(w, mode="horizon", checkpoint_every=20, objective="time_average")
        g2, r2 = s.gradient(w, mode="horizon", checkpoint_every=20, objective="time_average",
                            record_budget_bytes=6 * rec_bytes)
    assert r2.forward_recomputed > r1.forward_recomputed
    assert rel_l2(g2, g1) < 1e-6


@pytest.mark.gpu
def test_unsteady_driver_reports_every_schedule(gpu_lib):
    """The K-sweep driver on a small pulsatile grid: every schedule reports its
    memory and recomputation, and all of them give the same gradient."""
    from implexity_b200 import unsteady

    logs = []
    base, recs = unsteady.run((12, 8, 6), 40, [10, 40], period_steps=16, snapshots=(3,), log=logs.append)
    assert base["objective_time_average"] > 0.0
    assert [r.get("K", r.get("binomial_snapshots")) for r in recs] == [10, 40, 3]
    for r in recs:
        assert r["adjoint_steps"] == 40
        assert r["peak_state_GB"] > 0.0
        assert r["grad_rel_l2_vs_first_K"] < 1e-5
    assert recs[2]["forward_recomputed"] > recs[0]["forward_recomputed"]
    assert len(logs) == 1 + len(recs)


@pytest.mark.gpu
def test_fp16_time_average_close_to_fp32(gpu_lib):
    """16-bit storage through the fused response sums and the stage adjoint:
    time average and gradient within the format's resolution of FP32."""
    out = {}
    for storage in ("float32", "float16"):
        prob = workloads.pulsatile_problem(shape=(10, 7, 6), steps=40, lattice="D3Q19", u_mean=0.04, amp_frac=0.5,
                                           period_steps=16, ramp_steps=6, box_half_width=1, storage=storage)
        raw = workloads.uniform_design((10, 7, 6), 2)
        with LbmSolver(prob) as s:
            s.set_design(raw)
            s.forward()
            avg = s.time_average()
            g, _ = s.gradient(workloads.objective_weights(), mode="horizon", checkpoint_every=10,
                              objective="time_average", lambda_storage=storage)
        out[storage] = (avg, g)
    (a32, g32), (a16, g16) = out["float32"], out["float16"]
    for k in (3, 6, 7):
        assert abs(a16[k] - a32[k]) <= 5e-3 * abs(a32[k]), (k, a16[k], a32[k])
    assert rel_l2(g16, g32) < 5e-3, rel_l2(g16, g32)
