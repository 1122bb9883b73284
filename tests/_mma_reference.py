"""numpy restatement of the reference optimiser's MMA and GCMMA steps
(crates/implexity-optim/src/mma.rs) for one constraint, test
infrastructure for tests/test_mma_one_step.py and tests/test_gcmma.py.

The pieces follow the reference routine by routine: asymptote_update
(:522-553), trust_box (:555-571), pq / big_pq (:573-615), rhs (:617-622),
psi_rows (:624-629), step (:633-662) and step_gcmma (:666-769).  The
subproblem, which the reference solves with a primal-dual interior-point
method stopping at epsimin = 1e-7 (solve_subproblem, :906), is solved here
exactly through its one-dimensional dual: with a = 0 the artificial variable
z is 0 and, for one constraint,
    min  sum_i P_i / (u_i - x_i) + Q_i / (x_i - l_i) + c y + y^2 d / 2
    s.t. sum_i p_i / (u_i - x_i) + q_i / (x_i - l_i) - y <= b,  alpha <= x <= beta,  y >= 0
has, for a multiplier lam >= 0, the Lagrangian minimiser
    x_i = clip((sqrt(p0_i + lam p_i) l_i + sqrt(q0_i + lam q_i) u_i) / (sqrt(...) + sqrt(...)), alpha_i, beta_i),
    y = max(0, (lam - c) / d),
and the constraint residual decreases in lam, so lam follows by bisection.
"""
import numpy as np

# MmaOptions::default (mma.rs:107-129), MmaOptimizer::new's c = 1000, d = 1,
# GcmmaOptions::default (mma.rs:139-145)
MOVE, A_INIT, A_EXP, A_CON, A_LO, A_HI, RAA0, ALBEFA, C, D, EPSIMIN = (0.2, 0.5, 1.2, 0.7, 0.01, 10.0, 1e-5, 0.1,
                                                                       1000.0, 1.0, 1e-7)
RHO_MIN, RHO_INIT, RHO_GROWTH, MAX_CONSERVATIVE = 1e-6, 0.1, 10.0, 15


def begin(state, xk, xkm1, xkm2, xmin, xmax):
    """Asymptotes (stored in state) and the move box of one step."""
    span = xmax - xmin
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
    return l, u, alpha, beta


def pq(df, rho, xk, l, u, xmami):
    dfp, dfm = np.maximum(df, 0.0), np.maximum(-df, 0.0)
    r = 0.001 * (dfp + dfm) + rho / xmami
    return (dfp + r) * (u - xk) ** 2, (dfm + r) * (xk - l) ** 2


def psi(p, q, x, l, u):
    return float(np.sum(p / (u - x)) + np.sum(q / (x - l)))


def solve_dual(p0, q0, p, q, b, l, u, alpha, beta):
    """The subproblem's exact solution (x, lam)."""
    def x_of(lam):
        sp, sq = np.sqrt(p0 + lam * p), np.sqrt(q0 + lam * q)
        return np.clip((sp * l + sq * u) / (sp + sq), alpha, beta)

    def residual(lam):
        return psi(p, q, x_of(lam), l, u) - max(0.0, (lam - C) / D) - b

    lam = 0.0
    if residual(0.0) > 0.0:
        lo, hi = 0.0, 1.0
        while residual(hi) > 0.0:
            hi *= 2.0
        for _ in range(200):
            mid = 0.5 * (lo + hi)
            lo, hi = (mid, hi) if residual(mid) > 0.0 else (lo, mid)
        lam = 0.5 * (lo + hi)
    return x_of(lam), lam


def mma_step(state, xk, xkm1, xkm2, df0, f1, df1, xmin=0.0, xmax=1.0):
    span = np.broadcast_to(np.asarray(xmax - xmin, float), xk.shape)
    xmami = np.maximum(span, 1e-5)
    l, u, alpha, beta = begin(state, xk, xkm1, xkm2, xmin, xmax)
    p0, q0 = pq(df0, RAA0, xk, l, u, xmami)
    p, q = pq(df1, RAA0, xk, l, u, xmami)
    b = psi(p, q, xk, l, u) - f1
    x, lam = solve_dual(p0, q0, p, q, b, l, u, alpha, beta)
    state["iter"] = state.get("iter", 0) + 1
    return x, lam


def gcmma_step(state, xk, xkm1, xkm2, f0, df0, f1, df1, eval_true, xmin=0.0, xmax=1.0):
    """One GCMMA step; returns x, lam, inner iterations, conservative, (rho0, rho)."""
    span = np.broadcast_to(np.asarray(xmax - xmin, float), xk.shape)
    xmami = np.maximum(span, 1e-5)
    n = xk.size
    l, u, alpha, beta = begin(state, xk, xkm1, xkm2, xmin, xmax)
    rho0 = max(RHO_MIN, RHO_INIT * float(np.sum(np.abs(df0) * span)) / n)
    rho = max(RHO_MIN, RHO_INIT * float(np.sum(np.abs(df1) * span)) / n)
    inner, conservative = 0, False
    while True:
        p0, q0 = pq(df0, rho0, xk, l, u, xmami)
        p, q = pq(df1, rho, xk, l, u, xmami)
        b = psi(p, q, xk, l, u) - f1
        x, lam = solve_dual(p0, q0, p, q, b, l, u, alpha, beta)
        r0 = f0 - psi(p0, q0, xk, l, u)
        f0app = r0 + psi(p0, q0, x, l, u)
        fapp = psi(p, q, x, l, u) - b
        f0new, f1new = eval_true(x)
        bad0 = f0app + EPSIMIN < f0new
        bad1 = fapp + EPSIMIN < f1new
        if not (bad0 or bad1):
            conservative = True
            break
        if inner >= MAX_CONSERVATIVE:
            break
        inner += 1
        w = max(float(np.sum((x - xk) / (u - x) * ((x - xk) / (x - l)) * ((u - l) / xmami))), 1e-12)
        if bad0:
            rho0 = min(1.1 * (rho0 + (f0new - f0app) / w), RHO_GROWTH * rho0)
        if bad1:
            rho = min(1.1 * (rho + (f1new - fapp) / w), RHO_GROWTH * rho)
    state["iter"] = state.get("iter", 0) + 1
    return x, lam, inner, conservative, (rho0, rho)
