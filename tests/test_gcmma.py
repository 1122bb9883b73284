"""GCMMA, the conservative variant of the host MMA (mma_enable_gcmma /
mma_step_gcmma, restating MmaOptimizer::gcmma and step_gcmma of
crates/implexity-optim/src/mma.rs:339-355, 666-769).

- The reference's options and contract messages.
- Steps at n = 1000 against the numpy restatement of step_gcmma
  (tests/_mma_reference.py, exact dual subproblem solve) on a strongly
  curved objective whose plain MMA approximation is not conservative: the same
  number of conservative inner iterations, the same rho growth, and the
  trial point within the interior-point tolerance (bars as in
  tests/test_mma_one_step.py).
- Convergence to the KKT point of a two-constraint quadratic with every
  accepted approximation conservative.
"""
import numpy as np
import pytest
from _mma_reference import gcmma_step as reference_gcmma_step

from implexity_b200 import mma
from implexity_b200.problem import ContractError


def test_default_options_match_reference():
    g = mma.default_gcmma_options()
    assert g == {"rho_min": 1e-6, "rho_init": 0.1, "rho_growth": 10.0, "max_conservative": 15}


def test_contract_messages():
    with pytest.raises(ContractError, match="rho_growth > 1"):
        mma.MmaOptimizer(3, 1, gcmma={"rho_growth": 1.0})
    with pytest.raises(ContractError, match="max_conservative must be >= 0"):
        mma.MmaOptimizer(3, 1, gcmma={"max_conservative": -1})
    opt = mma.MmaOptimizer(3, 1, gcmma=True)
    x = np.full(3, 0.5)
    with pytest.raises(ContractError, match="GCMMA.step requires eval_true"):
        opt.step(x, x, x, 1.0, np.ones(3), [0.0], np.ones((1, 3)))
    with pytest.raises(ContractError, match="expected 1"):
        opt.step_gcmma(x, x, x, 1.0, np.ones(3), [0.0], np.ones((1, 3)), lambda v: (1.0, [0.0, 0.0]))


def test_eval_true_exception_propagates():
    opt = mma.MmaOptimizer(3, 1, gcmma=True)
    x = np.full(3, 0.5)

    def boom(v):
        raise ValueError("solver refused")

    with pytest.raises(ValueError, match="solver refused"):
        opt.step_gcmma(x, x, x, 1.0, np.ones(3), [0.0], np.ones((1, 3)), boom)


def _curved(n, seed):
    """f0 = sum_i a_i x_i + 4 sum_i (x_i - 0.5)^2 (more curvature than the
    MMA approximation has at the first rho: its value at the trial point is
    underestimated), f1 = mean(x) - 0.45."""
    a = np.random.default_rng(seed).uniform(-1.0, 1.0, n)

    def true(x):
        return float(a @ x + 4.0 * np.sum((x - 0.5) ** 2)), float(x.mean() - 0.45)

    def grads(x):
        return a + 8.0 * (x - 0.5), np.full(n, 1.0 / n)

    return true, grads


@pytest.mark.parametrize("seed", [0, 1])
def test_step_matches_numpy_restatement(seed):
    n = 1000
    true, grads = _curved(n, seed)
    opt = mma.MmaOptimizer(n, 1, x_min=0.0, x_max=1.0, gcmma=True)
    state = {}
    x = np.random.default_rng(seed + 10).uniform(0.3, 0.7, n)
    xm1 = xm2 = x.copy()
    inners = []
    for it in range(3):
        f0, f1 = true(x)
        g0, g1 = grads(x)
        x_ref, lam_ref, inner_ref, cons_ref, rho_ref = reference_gcmma_step(
            state, x, xm1, xm2, f0, g0, f1, g1, lambda v: true(v))
        x_new = opt.step_gcmma(x, xm1, xm2, f0, g0, [f1], g1[None, :], lambda v: (true(v)[0], [true(v)[1]]))
        info = opt.last
        assert info.inner_iterations == inner_ref and info.conservative == cons_ref, (it, info, inner_ref)
        rho = opt.gcmma_state()["rho"]
        np.testing.assert_allclose(rho, rho_ref, rtol=1e-3)
        d = np.abs(x_new - x_ref)
        assert np.median(d) <= 2e-6 and np.quantile(d, 0.99) <= 1e-4 and d.max() <= 1e-2, (it, d.max())
        assert abs(float(opt.dual_variables()[0]) - lam_ref) <= 1e-4 * lam_ref + 1e-4
        inners.append(inner_ref)
        xm2, xm1, x = xm1, x, x_new
    assert max(inners) >= 1  # the plain approximation was not conservative somewhere


def test_two_constraint_quadratic_reaches_kkt_point():
    # min |x|^2  s.t.  |x - (5,2,1)|^2 <= 9,  |x - (3,4,3)|^2 <= 9,  0 <= x <= 5
    c1, c2 = np.array([5.0, 2.0, 1.0]), np.array([3.0, 4.0, 3.0])

    def true(x):
        return float(x @ x), [float((x - c1) @ (x - c1) - 9.0), float((x - c2) @ (x - c2) - 9.0)]

    opt = mma.MmaOptimizer(3, 2, x_min=0.0, x_max=5.0, gcmma=True)
    x = np.array([4.0, 3.0, 2.0])
    xm1 = xm2 = x.copy()
    for _ in range(40):
        f0, fs = true(x)
        dfs = np.stack([2 * (x - c1), 2 * (x - c2)])
        xn = opt.step_gcmma(x, xm1, xm2, f0, 2 * x, fs, dfs, true)
        assert opt.last.conservative
        xm2, xm1, x = xm1, x, xn
    f0, fs = true(x)
    assert max(fs) <= 1e-5
    assert opt.kkt_residual(x, 2 * x, fs, np.stack([2 * (x - c1), 2 * (x - c2)])) < 1e-4
    np.testing.assert_allclose(x, [2.0175, 1.7800, 1.2375], atol=2e-3)
