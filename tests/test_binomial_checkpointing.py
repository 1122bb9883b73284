"""Binomial (revolve) checkpointing of the horizon adjoint.

The schedule restates BinomialSchedule (implexity-ad/src/revolve.rs:128-283).
CPU: its forward-step count equals the closed form of optimal_forward_steps
(revolve.rs:90-125) and an independent dynamic program over all split points
(the minimum over m of m + A(l - m, s - 1) + A(m, s)), and its peak equals the
slots given, capped by what the chain can use.  GPU: the gradient through the
binomial schedule equals the Every(K) gradient (1e-6, FP32 rescaling order)
and the oracle's (1e-4), for the final and the time-averaged objective.
"""
from functools import lru_cache
from math import comb

import numpy as np
import pytest

from implexity_b200 import LbmSolver, normalize, workloads
from implexity_b200.problem import ContractError
from implexity_b200.solver import binomial_plan
from oracle.oracle import Oracle


def closed_form(steps, slots):
    if steps <= 1:
        return steps
    r = 0
    while comb(slots + r, r) < steps:
        r += 1
    return r * steps - comb(slots + r, r) * r // (slots + 1) + 1


@lru_cache(maxsize=None)
def advances(length, slots):
    """Fewest advanced steps to reverse `length` steps from a held start."""
    if length <= 1:
        return 0
    if slots == 1:
        return length * (length - 1) // 2
    return min(m + advances(length - m, slots - 1) + advances(m, slots) for m in range(1, length))


@pytest.mark.parametrize("steps,slots", [(1, 1), (2, 1), (7, 1), (10, 3), (25, 2), (40, 4), (60, 5), (33, 33), (64, 6)])
def test_plan_is_optimal(steps, slots):
    fw, peak = binomial_plan(steps, slots)
    assert fw == closed_form(steps, slots)
    assert fw == advances(steps, slots) + 1
    assert 1 <= peak <= slots


@pytest.mark.parametrize("steps,slots", [(4000, 10), (4000, 60), (100000, 20), (5000, 1)])
def test_large_plans(steps, slots):
    fw, peak = binomial_plan(steps, slots)
    assert fw == closed_form(steps, slots)
    assert peak <= slots


def test_plan_contract():
    with pytest.raises(ContractError):
        binomial_plan(10, 0)
    with pytest.raises(ContractError):
        binomial_plan(0, 3)


def small(steps=40, time_average=False):
    if time_average:
        prob = workloads.pulsatile_problem(shape=(10, 7, 6), steps=steps, lattice="D3Q19", u_mean=0.04, amp_frac=0.5,
                                           period_steps=16, ramp_steps=6, box_half_width=1)
    else:
        prob = workloads.channel_problem(shape=(12, 8, 6), steps=steps, collision="trt")
    norm = normalize(prob)
    return norm, workloads.uniform_design(norm.shape, 5)


@pytest.mark.gpu
@pytest.mark.parametrize("objective", ["final", "time_average"])
@pytest.mark.parametrize("snapshots", [1, 3, 8])
def test_binomial_gradient_matches_every_k_and_oracle(gpu_lib, objective, snapshots):
    steps = 40
    norm, raw = small(steps, objective == "time_average")
    w = workloads.objective_weights()
    o = Oracle(norm)
    mode = "time_average" if objective == "time_average" else "horizon"
    g_ref, _, _, st = o.gradient(raw, w, mode=mode, K=10)
    assert st == 0
    with LbmSolver(norm) as s:
        s.set_design(raw)
        g_k, r_k = s.gradient(w, mode="horizon", checkpoint_every=10, objective=objective)
        g_b, r_b = s.gradient(w, mode="horizon", checkpointing="binomial", snapshots=snapshots, objective=objective)
        cells = s.cells
    fw, peak = binomial_plan(steps, snapshots)
    assert r_b.iterations == steps
    assert r_b.forward_recomputed == fw - steps
    # the slots held, plus one record slot
    assert r_b.peak_state_bytes >= peak * cells * 19 * 4
    assert np.linalg.norm(g_b - g_k) <= 1e-6 * np.linalg.norm(g_k)
    assert np.linalg.norm(g_b.ravel() - g_ref.ravel()) <= 1e-4 * np.linalg.norm(g_ref)


@pytest.mark.gpu
def test_binomial_needs_a_snapshot(gpu_lib):
    norm, raw = small(10)
    with LbmSolver(norm) as s:
        s.set_design(raw)
        with pytest.raises(ContractError, match="snapshot"):
            s.gradient(workloads.objective_weights(), checkpointing="binomial", snapshots=0)
