"""The host MMA step (include/mma_cpu.h) against an independent numpy
restatement of one MmaOptimizer::step (crates/implexity-optim/src/mma.rs:
633-662) at n = 1000, m = 1 (tests/_mma_reference.py): the asymptotes (the
initial ones for the first two steps and the adaptive update after), the
move box, the p/q coefficients and the right-hand side are restated
directly; the subproblem, which the reference solves with a primal-dual
interior-point method stopping at epsimin = 1e-7, is solved exactly through
its one-dimensional dual.

Bars: the interior-point solution sits within its own stopping tolerance of
the exact one -- median |dx| <= 2e-6 and 99th percentile <= 1e-4; the few
coordinates further off (at most 1%, none by more than 1e-2) have their
exact optimum on or next to a bound of the move box, where the barrier term
epsimin / (x - alpha) of the last interior-point level holds the iterate
about sqrt(epsimin / curvature) away, up to ~1e-2 where the subproblem is
flat (the reference's own subproblem KKT measure stays ~2e-4 there); the
multiplier agrees within 1e-4 relative (plus 1e-4 absolute when the
constraint is inactive).  A wrong asymptote, box or coefficient moves x by
1e-2 or more in the interior.
"""
import numpy as np
import pytest
from _mma_reference import mma_step as reference_step

from implexity_b200 import mma


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
