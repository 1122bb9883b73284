"""The host MMA step (include/mma_cpu.h) against an independent numpy
restatement of one MmaOptimizer::step (crates/implexity-optim/src/mma.rs:
633-662) at n = 1000, m = 1: the asymptotes (asymptote_update, :522-550, the
initial ones for the first two steps and the adaptive update after), the
move box (trust_box, :553-569), the p/q coefficients (pq / big_pq, :572-604)
and the right-hand side (rhs, :613-618) are restated directly; the
subproblem, which the reference solves with a primal-dual interior-point
method stopping at epsimin = 1e-7 (solve_subproblem, :906), is solved here
exactly through its one-dimensional dual.

With a = 0 the artificial variable z is 0 and, for one constraint, the
subproblem is
    min  sum_i P_i / (u_i - x_i) + Q_i / (x_i - l_i) + c y + y^2 d / 2
    s.t. sum_i p_i / (u_i - x_i) + q_i / (x_i - l_i) - y <= b,  alpha <= x <= beta,  y >= 0,
whose Lagrangian minimiser for a multiplier lam >= 0 is
    x_i = clip((sqrt(p0_i + lam p_i) l_i + sqrt(q0_i + lam q_i) u_i) / (sqrt(...) + sqrt(...)), alpha_i, beta_i),
    y = max(0, (lam - c) / d);
the constraint residual is decreasing in lam, so lam follows by bisection.

Bars: the interior-point solution sits within its own stopping tolerance of
the exact one -- median |dx| <= 2e-6 and 99th percentile <= 1e-4; the few
coordinates further off (at most 1%, none by more than 1e-2) have their
exact optimum on or next to a bound of the move box, where the barrier term
epsimin / (x - alpha) of the last interior-point level holds the iterate
about sqrt(epsimin / curvature) away, up to ~1e-2 where the subproblem is
flat (the reference's own subproblem KKT measure stays ~2e-4 there); the multiplier
agrees within 1e-4 relative (plus 1e-4 absolute when the constraint is
inactive).  A wrong asymptote, box or coefficient moves x by 1e-2 or more
in the interior.
"""
import numpy as np
import pytest

from implexity_b200 import mma

# MmaOptions::default (mma.rs:107-129) and the constraint coefficients of MmaOptimizer::new (c = 1000, d = 1)
MOVE, A_INIT, A_EXP, A_CON, A_LO, A_HI, RAA0, ALBEFA, C, D = 0.2, 0.5, 1.2, 0.7, 0.01, 10.0, 1e-5, 0.1, 1000.0, 1.0


def reference_step(state, xk, xkm1, xkm2, df0, f1, df1, xmin, xmax):
    span = xmax - xmin
    xmami = np.maximum(span, 1e-5)
    if state.get("iter", 0) >= 2:
        zzz = (xk - xkm1) * (xkm1 - xkm2)
        factor = np.where(zzz > 0, A_EXP, np.where(zzz < 0, A_CON, 1.0))
        lo = xk - factor * (xkm1 - state["l"])
        up = xk + factor * (state["u"] - xkm1)
        l = np.minimum(np.maximum(lo, xk - A_HI * span), xk - A_LO * span)
        u = np.maximum(np.minimum(up, xk + A_HI * span), xk + A_LO * span)
    else:
        l, u = xk - A_INIT * span, xk + A_INIT * span
    state["l"], state["u"] = l, u
    alpha = np.maximum(np.maximum(l + ALBEFA * (xk - l), xk - MOVE * span), xmin)
    beta = np.minimum(np.minimum(u - ALBEFA * (u - xk), xk + MOVE * span), xmax)

    def pq(df):
        dfp, dfm = np.maximum(df, 0.0), np.maximum(-df, 0.0)
        r = 0.001 * (dfp + dfm) + RAA0 / xmami
        return (dfp + r) * (u - xk) ** 2, (dfm + r) * (xk - l) ** 2

    p0, q0 = pq(df0)
    p, q = pq(df1)
    b = np.sum(p / (u - xk)) + np.sum(q / (xk - l)) - f1

    def x_of(lam):
        sp, sq = np.sqrt(p0 + lam * p), np.sqrt(q0 + lam * q)
        return np.clip((sp * l + sq * u) / (sp + sq), alpha, beta)

    def residual(lam):
        x = x_of(lam)
        return np.sum(p / (u - x)) + np.sum(q / (x - l)) - max(0.0, (lam - C) / D) - b

    lam = 0.0
    if residual(0.0) > 0.0:
        lo, hi = 0.0, 1.0
        while residual(hi) > 0.0:
            hi *= 2.0
        for _ in range(200):
            mid = 0.5 * (lo + hi)
            lo, hi = (mid, hi) if residual(mid) > 0.0 else (lo, mid)
        lam = 0.5 * (lo + hi)
    state["iter"] = state.get("iter", 0) + 1
    x = x_of(lam)
    return x, lam


@pytest.mark.parametrize("seed", [0, 1])
@pytest.mark.parametrize("volume", [0.3, 0.7])
def test_step_matches_exact_subproblem_solution(seed, volume):
    n = 1000
    rng = np.random.default_rng(seed)
    opt = mma.MmaOptimizer(n, 1, x_min=0.0, x_max=1.0)
    state = {}
    x = rng.uniform(0.2, 0.8, n)
    xm1 = xm2 = x.copy()
    for it in range(4):
        df0 = rng.standard_normal(n) * rng.uniform(0.5, 1.5, n)
        f1 = float(x.mean() - volume)
        df1 = np.full(n, 1.0 / n)
        x_ref, lam_ref = reference_step(state, x, xm1, xm2, df0, f1, df1, 0.0, 1.0)
        x_new = opt.step(x, xm1, xm2, 1.0, df0, np.array([f1]), df1[None, :])
        d = np.abs(x_new - x_ref)
        assert np.median(d) <= 2e-6, (it, np.median(d))
        assert np.quantile(d, 0.99) <= 1e-4, (it, np.quantile(d, 0.99))
        far = d > 1e-4
        assert far.sum() <= n // 100, (it, far.sum())
        assert d.max() <= 1e-2, (it, d.max())
        assert opt.last.subproblem_converged
        lam = float(opt.dual_variables()[0])
        assert abs(lam - lam_ref) <= 1e-4 * lam_ref + 1e-4, (it, lam, lam_ref)
        xm2, xm1, x = xm1, x, x_new
