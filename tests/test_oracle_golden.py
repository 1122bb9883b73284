"""The FP64 oracle against the independent numpy restatement's golden
fixtures (tests/golden/make_golden.py): the reference's own problem template
(provider.rs:74-90) with BGK, and a ported TRT channel with a solid cell."""
import numpy as np
import pytest

from implexity_b200 import normalize
from oracle.oracle import Oracle

from _problems import golden_problem, load_golden

CASES = ["template_bgk", "channel_trt"]


@pytest.fixture(scope="module", params=CASES)
def case(request):
    name = request.param
    g = load_golden(name)
    norm = normalize(golden_problem(name))
    return name, g, norm, Oracle(norm)


def test_design_map(case):
    _, g, _, o = case
    phi, alpha = o.design(g["raw"])
    np.testing.assert_allclose(phi, g["phi"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(alpha, g["alpha"], rtol=1e-13, atol=1e-16)


def test_trajectory(case):
    _, g, norm, o = case
    f, d, mass, exch = o.history_trace(g["alpha"], norm.step_count)
    np.testing.assert_allclose(f, g["final"], rtol=0, atol=1e-14)
    np.testing.assert_allclose(mass, g["mass"], rtol=1e-13)
    np.testing.assert_allclose(exch[1:], g["exchange"], rtol=1e-10, atol=1e-13)
    assert d.nonfinite == 0


def test_responses(case):
    _, g, _, o = case
    r = o.vector(g["phi"], g["alpha"], g["final"])
    np.testing.assert_allclose(r, g["responses"], rtol=1e-9, atol=1e-12 * np.abs(g["responses"]).max())


@pytest.mark.parametrize("K", [0, 3])
def test_adjoint_gradient_matches_finite_differences(case, K):
    _, g, norm, o = case
    grad, resp, rep, st = o.gradient(g["raw"], g["weights"], mode="horizon", K=K)
    assert st == 0
    assert rep.iterations == norm.step_count
    cells = g["fd_cells"]
    scale = np.max(np.abs(g["fd_grad"]))
    np.testing.assert_allclose(grad[cells], g["fd_grad"], rtol=0, atol=1e-10 * scale)
