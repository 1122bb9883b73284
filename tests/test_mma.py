"""The host MMA (include/mma_cpu.h, restating MmaOptimizer of the reference
optimiser, crates/implexity-optim/src/mma.rs) on problems with known
optima: convergence to a KKT point of a two-constraint quadratic problem, a
volume-constrained linear problem whose solution is the top-weight cells,
and the reference's contract messages."""
import ctypes as C

import numpy as np
import pytest

from implexity_b200 import mma
from implexity_b200.problem import ContractError


def test_library_exports_every_header_symbol():
    lib = mma.load()
    for name in mma.EXPORTS:
        assert hasattr(lib, name), name


def test_default_options_match_reference():
    o = mma.default_options()
    assert o["move_limit"] == 0.2 and o["asymptote_init"] == 0.5 and o["asymptote_expand"] == 1.2
    assert o["asymptote_contract"] == 0.7 and o["asymptote_lo"] == 0.01 and o["asymptote_hi"] == 10.0
    assert o["raa0"] == 1e-5 and o["albefa"] == 0.1 and o["epsimin"] == 1e-7 and o["max_inner"] == 200


def _solve(opt, x, fun, iters):
    xm1 = xm2 = x.copy()
    for _ in range(iters):
        f0, g0, fs, gs = fun(x)
        xn = opt.step(x, xm1, xm2, f0, g0, fs, gs)
        xm2, xm1, x = xm1, x, xn
    return x


def test_two_constraint_quadratic_reaches_kkt_point():
    # min |x|^2  s.t.  |x - (5,2,1)|^2 <= 9,  |x - (3,4,3)|^2 <= 9,  0 <= x <= 5
    c1, c2 = np.array([5.0, 2.0, 1.0]), np.array([3.0, 4.0, 3.0])

    def fun(x):
        fs = np.array([np.sum((x - c1) ** 2) - 9.0, np.sum((x - c2) ** 2) - 9.0])
        gs = np.stack([2 * (x - c1), 2 * (x - c2)])
        return float(x @ x), 2 * x, fs, gs

    opt = mma.MmaOptimizer(3, 2, x_min=0.0, x_max=5.0)
    x = _solve(opt, np.array([4.0, 3.0, 2.0]), fun, 40)
    f0, g0, fs, gs = fun(x)
    lam = opt.dual_variables()
    assert np.all(fs <= 1e-6)
    assert np.all(lam >= -1e-12)
    # stationarity of the Lagrangian and complementary slackness
    assert np.linalg.norm(g0 + gs.T @ lam) < 1e-4 * np.linalg.norm(g0)
    assert np.all(np.abs(lam * fs) < 1e-6)
    assert opt.kkt_residual(x, g0, fs, gs.ravel()) < 1e-4


def test_volume_constrained_linear_problem_selects_top_weights():
    rng = np.random.default_rng(0)
    n = 1000
    w = rng.uniform(0.5, 1.5, n)

    def fun(x):
        return -float(w @ x) / n, -w / n, np.array([x.mean() - 0.4]), np.full((1, n), 1.0 / n)

    opt = mma.MmaOptimizer(n, 1, x_min=0.0, x_max=1.0)
    x = _solve(opt, np.full(n, 0.3), fun, 60)
    top = np.argsort(-w)[: int(0.4 * n)]
    target = np.zeros(n)
    target[top] = 1.0
    assert x.mean() <= 0.4 + 1e-6
    assert np.mean(np.abs(x - target)) < 2e-2


def test_contract_messages():
    with pytest.raises(ContractError, match="move_limit must lie in"):
        mma.MmaOptimizer(4, 1, move_limit=1.5)
    with pytest.raises(ContractError, match="x_max must exceed x_min"):
        mma.MmaOptimizer(2, 0, x_min=[0.0, 1.0], x_max=[1.0, 1.0])
    opt = mma.MmaOptimizer(2, 0)
    with pytest.raises(ContractError, match="outside"):
        opt.step(np.array([0.5, 1.5]), np.zeros(2), np.zeros(2), 1.0, np.ones(2))
    with pytest.raises(ContractError, match="non-finite entries in df0dx"):
        opt.step(np.array([0.5, 0.5]), np.zeros(2), np.zeros(2), 1.0, np.array([np.nan, 1.0]))
