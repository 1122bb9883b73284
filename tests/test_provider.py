"""The host mirror of LbmOperations (provider.py; design_ops.rs:41-58 as
implemented by provider.rs:374-461): input contracts on CPU, and on the GPU
evaluate_value / sensitivities_value / candidate admission against the oracle."""
import numpy as np
import pytest

from implexity_b200 import workloads
from implexity_b200.problem import ContractError
from implexity_b200.provider import (COORDINATE, LatticeBoltzmannProvider, _check_responses, _single_coordinate,
                                     design_identity)
from implexity_b200.solver import RESPONSES
from implexity_b200 import normalize
from oracle.oracle import Oracle


def test_design_and_response_contracts():
    with pytest.raises(ContractError, match="LBM requires exactly model:control"):
        _single_coordinate({"other": np.zeros(3)})
    with pytest.raises(ContractError, match="LBM requires exactly model:control"):
        _single_coordinate({COORDINATE: np.zeros(3), "x": np.zeros(3)})
    for bad in ([], ["nope"], ["pressure_drop_Pa", "pressure_drop_Pa"]):
        with pytest.raises(ContractError, match="Unknown, duplicated or empty LBM responses"):
            _check_responses(bad)
    _check_responses(["pressure_drop_Pa", "viscous_dissipation_W"])


def test_design_identity_is_a_content_hash():
    a = {COORDINATE: np.linspace(0, 1, 24).reshape(2, 3, 4)}
    b = {COORDINATE: np.linspace(0, 1, 24).reshape(2, 3, 4)}
    assert design_identity(a) == design_identity(b)
    b[COORDINATE][0, 0, 0] += 1e-12
    assert design_identity(a) != design_identity(b)


def test_invalid_problem_is_refused_before_any_device_work():
    prob = workloads.channel_problem(shape=(10, 8, 6), steps=5, collision="trt")
    prob["periodic_axes"] = [True, False, False]
    out = LatticeBoltzmannProvider().candidate_admission(prob, {COORDINATE: np.full((10, 8, 6), 0.5)},
                                                         {COORDINATE: np.full((10, 8, 6), 0.5)})
    assert out["allow"] is False and "periodic face cannot be a port" in out["reason"]


def small():
    prob = workloads.channel_problem(shape=(14, 9, 8), steps=40, collision="trt")
    raw = workloads.uniform_design((14, 9, 8), 2)
    return prob, raw


@pytest.mark.gpu
def test_evaluate_value_matches_oracle(gpu_lib):
    prob, raw = small()
    ev = LatticeBoltzmannProvider().evaluate_value(prob, {COORDINATE: raw})
    norm = normalize(prob)
    _, r_ref, _, st = Oracle(norm).gradient(raw, workloads.objective_weights(), mode="horizon", K=8)
    assert st == 0
    assert list(ev["responses"]) == RESPONSES
    for k in (0, 3, 4, 5, 6, 7):
        v = ev["responses"][RESPONSES[k]]
        assert abs(v - r_ref[k]) <= 1e-5 * abs(r_ref[k]), (RESPONSES[k], v, r_ref[k])
    f = ev["fields"]
    assert f["density_kg_m3"].shape == (14, 9, 8) and f["velocity_m_s"].shape == (14, 9, 8, 3)
    assert f["fluid_fraction"].shape == (14, 9, 8)
    n = f["wall_link_positions_m"].shape[0]
    assert n > 0 and f["wall_link_gauge_force_N"].shape == (n, 3)
    assert "wall_load_convention" in ev["diagnostics"] and "method" in ev["diagnostics"]


@pytest.mark.gpu
def test_sensitivities_value_matches_oracle(gpu_lib):
    prob, raw = small()
    names = ["pressure_drop_Pa", "viscous_dissipation_W"]
    out = LatticeBoltzmannProvider().sensitivities_value(prob, {COORDINATE: raw}, names)
    o = Oracle(normalize(prob))
    for name in names:
        w = np.zeros(8)
        w[RESPONSES.index(name)] = 1.0
        g_ref, _, _, st = o.gradient(raw, w, mode="horizon", K=8)
        assert st == 0
        g = out["gradients"][name][COORDINATE]
        assert np.linalg.norm(g.ravel() - g_ref.ravel()) <= 1e-4 * np.linalg.norm(g_ref), name


@pytest.mark.gpu
def test_candidate_admission_allows_an_admitted_design(gpu_lib):
    prob, raw = small()
    out = LatticeBoltzmannProvider().candidate_admission(prob, {COORDINATE: raw}, {COORDINATE: raw})
    assert out["allow"] is True and out["diagnostics"]["relative_mass_drift"] < 1e-6
