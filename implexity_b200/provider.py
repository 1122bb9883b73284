"""``LatticeBoltzmannProvider``: the reference provider's operator interface over
the CUDA library.

Mirrors ``LbmOperations`` (crates/implexity-physics-lbm/src/design_ops.rs:41-58)
as implemented by ``LatticeBoltzmannProvider`` (src/provider.rs:374-461):

* ``preflight_value(problem, design)``  -> diagnostics mapping with ok/issues
* ``evaluate_value(problem, design)``    -> Evaluation (responses, diagnostics, fields)
* ``sensitivities_value(problem, design, responses)`` -> DesignSensitivities
* ``admission_value(problem, candidate)`` -> diagnostics

``problem`` is the JSON problem mapping (solver.rs:46-65) and ``design`` the
NamedArrays ``{"model:control": array}`` (provider.rs:55).  Errors are raised
as ``ContractError`` with the reference's messages.

The provider caches one ``LbmSolver`` (device buffers) per problem mapping so
that an optimiser that calls evaluate/sensitivities for many designs of one
problem reuses the same GPU allocation; the reference re-normalises per call
and so does this class (cheap compared with a trajectory).
"""
from __future__ import annotations

import hashlib
import json

import numpy as np

from .problem import ContractError, normalize
from .solver import RESPONSES, LbmSolver

NAME = "lattice_boltzmann_d3q19"
COORDINATE = "model:control"
UNITS = ["m/s", "m/s", "m/s", "J", "W", "m^3", "Pa", "W"]


def _single_coordinate(design) -> np.ndarray:
    # design_ops.rs:239-249
    if not isinstance(design, dict) or len(design) != 1 or COORDINATE not in design:
        raise ContractError("LBM requires exactly model:control")
    return np.asarray(design[COORDINATE], dtype=float)


def _check_responses(names) -> None:
    # design_ops.rs:229-236
    if not names or len(set(names)) != len(names) or any(n not in RESPONSES for n in names):
        raise ContractError("Unknown, duplicated or empty LBM responses")


def _key(problem) -> str:
    def enc(o):
        if isinstance(o, np.ndarray):
            return {"__nd__": o.tolist()}
        raise TypeError
    return json.dumps(problem, sort_keys=True, default=enc)


class LatticeBoltzmannProvider:
    IMPLEMENTATION = "implexity_b200.provider.LatticeBoltzmannProvider"

    def __init__(self):
        self._cache: dict[str, LbmSolver] = {}

    def _solver(self, problem) -> LbmSolver:
        norm = normalize(problem)
        key = _key(problem)
        s = self._cache.get(key)
        if s is None:
            self._cache.clear()
            s = LbmSolver(norm)
            self._cache[key] = s
        return s

    def _method(self, s: LbmSolver) -> dict:
        o = s.problem.options
        lat = f"D3Q{o.lattice}"
        return {
            "method": f"Independent {lat} {o.collision.upper()} / Guo / halfway bounce-back (CUDA sm_100a)",
            "method_version": f"{lat.lower()}-{o.collision}-guo-bounceback-porous-v1",
            "population_dtype": o.storage,
        }

    def parts(self, problem, design):
        """provider.rs:249-263: normalise, map the design, run the trajectory, admit."""
        raw = _single_coordinate(design)
        s = self._solver(problem)
        p = s.problem
        if raw.shape != p.shape or not np.all(np.isfinite(raw)) or np.any((raw < 0) | (raw > 1)):
            raise ContractError("model:control must be a finite shape-matched array in [0,1]")
        s.set_design(raw)
        d = s.forward()
        unit = p.density_kg_m3 * p.spacing_m**3
        diag = {
            "maximum_mach": d.maximum_mach,
            "relative_mass_drift": d.relative_mass_drift,
            "relaxation_time": d.relaxation_time,
            "physical_qualification": False,
            "steady_state_certified": False,
            "derivative_scope": "Discrete fixed-horizon porous-resistance trajectory; fixed walls and forcing",
            **self._method(s),
            "boundary_population_mass_exchange_total_kg": d.boundary_exchange_total * unit,
            "step_count": p.step_count,
            "end_time_s": p.step_count * p.step_s,
            "device_ms": d.device_ms,
            "field_metadata": {"shape": list(p.shape), "spacing_m": p.spacing_m, "origin_m": list(p.origin_m)},
        }
        return s, raw, diag

    # ---- LbmOperations
    def preflight_value(self, problem, design) -> dict:
        _, _, diag = self.parts(problem, design)
        return {"ok": True, "issues": [], **diag}

    def evaluate_value(self, problem, design) -> dict:
        s, _, diag = self.parts(problem, design)
        # fixed-wall momentum exchange of the last interval (provider.rs:312-321)
        loads = s.wall_loads(0.0)
        diag["wall_load_convention"] = (
            "Last interval fixed-wall momentum exchange, gauge datum zero; includes pressure and viscous effects, "
            "not a solved structural coupling"
        )
        values = s.responses()
        fields = s.fields()
        phi, _ = s.design()
        fields["fluid_fraction"] = phi
        if len(loads["wall_link_positions_m"]):  # insert_wall_fields (provider.rs:284-298)
            fields.update(loads)
        return {
            "provider": NAME,
            "responses": {n: float(v) for n, v in zip(RESPONSES, values)},
            "diagnostics": diag,
            "fields": fields,
        }

    def sensitivities_value(self, problem, design, responses) -> dict:
        _check_responses(list(responses))
        s, raw, diag = self.parts(problem, design)
        values = s.responses()
        o = s.problem.options
        out_values, gradients = {}, {}
        for name in responses:
            k = RESPONSES.index(name)
            w = np.zeros(len(RESPONSES))
            w[k] = 1.0
            if o.adjoint == "steady":
                g, rep = s.gradient(
                    w, mode="steady", lambda_storage=o.lambda_storage, tolerance=o.tolerance,
                    max_iterations=o.max_iterations,
                )
            else:
                # the horizon adjoint re-runs the trajectory from its checkpoints
                g, rep = s.gradient(w, mode="horizon", lambda_storage=o.lambda_storage,
                                    checkpoint_every=o.checkpoint_every)
            if not np.all(np.isfinite(g)):
                raise ContractError("Nonfinite LBM sensitivity")
            out_values[name] = float(values[k])
            gradients[name] = {COORDINATE: g}
            diag.setdefault("adjoint", {})[name] = rep.__dict__
        return {"responses": out_values, "gradients": gradients, "diagnostics": diag}

    def admission_value(self, problem, candidate) -> dict:
        return self.parts(problem, candidate)[2]

    def candidate_admission(self, problem, current, candidate) -> dict:
        """candidate_design_admission record (design_ops.rs:204-227)."""
        out = {
            "current_design_state_id": design_identity(current),
            "candidate_design_state_id": design_identity(candidate),
        }
        try:
            diag = self.admission_value(problem, candidate)
        except ContractError as e:
            out.update(allow=False, reason=str(e))
        else:
            out.update(allow=True, reason="Fixed LBM trajectory admitted", diagnostics=diag)
        return out


def design_identity(design) -> str:
    """Content hash of a NamedArrays design."""
    h = hashlib.sha256()
    for k in sorted(design):
        a = np.ascontiguousarray(design[k], dtype=np.float64)
        h.update(k.encode())
        h.update(str(a.shape).encode())
        h.update(a.tobytes())
    return h.hexdigest()


def sensitivity_design(provider: LatticeBoltzmannProvider, problem, design, response: str) -> dict:
    """design_ops.rs:61-71 single_sensitivity."""
    out = provider.sensitivities_value(problem, design, [response])
    return {
        "value": out["responses"].get(response, float("nan")),
        "gradients": out["gradients"].get(response, {}),
        "diagnostics": out["diagnostics"],
    }
