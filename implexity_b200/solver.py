"""Thin Python handle over the C-ABI (include/lbm_b200.h).

``LbmSolver`` owns one ``lbm_handle``: device buffers for one normalised
problem, reused across designs.  Every method is one C-ABI call; errors come
back as the exception type matching the library's status code.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from .problem import ContractError, NormalizedProblem, normalize

RESPONSES = [
    "mean_velocity_x_m_s",
    "mean_velocity_y_m_s",
    "mean_velocity_z_m_s",
    "kinetic_energy_J",
    "porous_dissipation_W",
    "fluid_volume_m3",
    "pressure_drop_Pa",
    "viscous_dissipation_W",
]


class LbmError(RuntimeError):
    status = -1


class ConvergenceError(LbmError):
    status = _abi.LBM_E_CONVERGENCE


class CudaError(LbmError):
    status = _abi.LBM_E_CUDA


class StateError(LbmError):
    status = _abi.LBM_E_STATE


def _raise(status: int, msg: str):
    if status == _abi.LBM_E_CONTRACT:
        raise ContractError(msg)
    cls = {_abi.LBM_E_CONVERGENCE: ConvergenceError, _abi.LBM_E_CUDA: CudaError, _abi.LBM_E_STATE: StateError}.get(
        status, LbmError
    )
    raise cls(msg)


def _choice(name: str, value: str, table: dict) -> int:
    if value not in table:
        raise ContractError(f"{name} must be one of {', '.join(table)} (got {value!r})")
    return table[value]


def _dp(a: np.ndarray | None):
    if a is None:
        return None
    return a.ctypes.data_as(C.POINTER(C.c_double))


@dataclass
class Diagnostics:
    maximum_mach: float
    relative_mass_drift: float
    relaxation_time: float
    minimum_population: float
    boundary_exchange_total: float
    steps: int
    admitted: bool
    device_ms: float
    nonfinite: bool = False

    @classmethod
    def of(cls, d: _abi.Diag) -> "Diagnostics":
        return cls(
            d.maximum_mach,
            d.relative_mass_drift,
            d.relaxation_time,
            d.minimum_population,
            d.boundary_exchange_total,
            int(d.steps),
            bool(d.admitted),
            d.device_ms,
            bool(d.nonfinite),
        )


@dataclass
class AdjointReport:
    residual: float
    iterations: int
    forward_recomputed: int
    peak_state_bytes: int
    converged: bool
    forward_ms: float
    adjoint_ms: float
    sensitivity_ms: float


def binomial_plan(steps: int, snapshots: int) -> tuple[int, int]:
    """(forward steps, peak snapshots) of the binomial checkpoint schedule
    (host only; implexity-ad/src/revolve.rs BinomialSchedule)."""
    fw, pk = C.c_int64(), C.c_int64()
    st = _abi.load().lbm_binomial_plan(int(steps), int(snapshots), C.byref(fw), C.byref(pk))
    if st != 0:
        raise ContractError(f"no binomial schedule for {steps} steps and {snapshots} snapshots")
    return int(fw.value), int(pk.value)


class LbmSolver:
    def __init__(self, problem: dict | NormalizedProblem):
        self.problem = problem if isinstance(problem, NormalizedProblem) else normalize(problem)
        self.lib = _abi.load()
        self._cp = self.problem.to_c()
        h = C.c_void_p()
        st = self.lib.lbm_create(C.byref(self._cp), C.byref(h))
        if st != _abi.LBM_OK:
            _raise(st, self.lib.lbm_last_error(None).decode())
        self.h = h
        info = _abi.Info()
        self.lib.lbm_info(self.h, C.byref(info))
        self.cells = int(info.cells)
        self.fluid_cells = int(info.fluid_cells)
        self.q = int(info.q)
        self.tau = float(info.tau)
        self.acceleration_lattice = tuple(info.acceleration_lattice)
        self.last_diag: Diagnostics | None = None

    # -- lifetime
    def close(self):
        if getattr(self, "h", None):
            self.lib.lbm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def _check(self, st: int):
        if st != _abi.LBM_OK:
            _raise(st, self.lib.lbm_last_error(self.h).decode())

    @property
    def shape(self):
        return self.problem.shape

    def device_bytes(self) -> int:
        info = _abi.Info()
        self.lib.lbm_info(self.h, C.byref(info))
        return int(info.device_bytes)

    # -- design
    def set_design(self, raw: np.ndarray):
        r = np.ascontiguousarray(raw, dtype=np.float64)
        if r.shape != tuple(self.shape):
            raise ContractError("model:control must be a finite shape-matched array in [0,1]")
        self._check(self.lib.lbm_set_design(self.h, _dp(r), r.size))

    def design(self) -> tuple[np.ndarray, np.ndarray]:
        phi = np.empty(self.shape)
        alpha = np.empty(self.shape)
        self._check(self.lib.lbm_get_design(self.h, _dp(phi), _dp(alpha)))
        return phi, alpha

    # -- forward
    def forward(self, steps: int = 0) -> Diagnostics:
        d = _abi.Diag()
        st = self.lib.lbm_forward(self.h, int(steps), C.byref(d))
        self.last_diag = Diagnostics.of(d)
        self._check(st)
        return self.last_diag

    def advance(self, steps: int) -> Diagnostics:
        d = _abi.Diag()
        st = self.lib.lbm_advance(self.h, int(steps), C.byref(d))
        self.last_diag = Diagnostics.of(d)
        self._check(st)
        return self.last_diag

    def trajectory(self) -> dict[str, np.ndarray]:
        """Per-state admission record of the last forward/advance."""
        n = (self.last_diag.steps if self.last_diag else 0) + 1
        out = {k: np.empty(n) for k in ("mass", "exchange", "min_population", "max_speed")}
        self._check(self.lib.lbm_trajectory(self.h, _dp(out["mass"]), _dp(out["exchange"]),
                                            _dp(out["min_population"]), _dp(out["max_speed"]), n))
        return out

    def set_populations(self, f: np.ndarray):
        a = np.ascontiguousarray(f, dtype=np.float64).reshape(-1)
        self._check(self.lib.lbm_set_populations(self.h, _dp(a), a.size))

    def populations(self) -> np.ndarray:
        out = np.empty(self.cells * self.q)
        self._check(self.lib.lbm_get_populations(self.h, _dp(out), out.size))
        return out.reshape(self.cells, self.q)

    def time_average(self) -> np.ndarray:
        """Responses averaged over the states 1..T of the last forward."""
        out = np.empty(_abi.N_RESPONSES)
        self._check(self.lib.lbm_time_average(self.h, _dp(out)))
        return out

    def responses(self) -> np.ndarray:
        out = np.empty(_abi.N_RESPONSES)
        self._check(self.lib.lbm_responses(self.h, _dp(out)))
        return out

    def wall_loads(self, pressure_datum_pa: float = 0.0) -> dict[str, np.ndarray]:
        """Fixed-wall momentum-exchange loads of the last interval: link
        midpoints [n,3] (m) and forces [n,3] (N), as evaluate_value's
        wall_link_positions_m / wall_link_gauge_force_N."""
        n = C.c_size_t(0)
        self._check(self.lib.lbm_wall_loads(self.h, 0.0, None, None, None, 0, C.byref(n)))
        pos = np.empty((n.value, 3))
        force = np.empty((n.value, 3))
        origin = np.ascontiguousarray(self.problem.origin_m, dtype=np.float64)
        self._check(self.lib.lbm_wall_loads(self.h, float(pressure_datum_pa), _dp(origin), _dp(pos), _dp(force),
                                            n.value, C.byref(n)))
        return {"wall_link_positions_m": pos, "wall_link_gauge_force_N": force}

    def fields(self) -> dict[str, np.ndarray]:
        rho = np.empty(self.shape)
        vel = np.empty(tuple(self.shape) + (3,))
        p = np.empty(self.shape)
        self._check(self.lib.lbm_fields(self.h, _dp(rho), _dp(vel), _dp(p)))
        return {"density_kg_m3": rho, "velocity_m_s": vel, "gauge_pressure_Pa": p}

    # -- adjoint
    def gradient(
        self,
        weights,
        mode: str = "horizon",
        lambda_storage: str = "float32",
        checkpoint_every: int = 0,
        tolerance: float = 1e-8,
        max_iterations: int = 100000,
        check_every: int = 50,
        objective: str = "final",
        record_budget_bytes: int = 0,
        checkpointing: str = "every",
        snapshots: int = 0,
    ) -> tuple[np.ndarray, AdjointReport]:
        """Design gradient of w . responses: of the final state (objective
        "final") or of their mean over the horizon's states ("time_average",
        horizon mode, problems with solver_options.time_average).  Horizon
        checkpointing is a state every `checkpoint_every` steps ("every") or
        the binomial schedule over `snapshots` states ("binomial")."""
        w = np.zeros(_abi.N_RESPONSES)
        w[: len(weights)] = np.asarray(weights, dtype=float)
        o = _abi.AdjointOpts()
        o.mode = _choice("mode", mode, {"horizon": _abi.LBM_ADJ_HORIZON, "steady": _abi.LBM_ADJ_STEADY})
        o.lambda_storage = _choice("lambda_storage", lambda_storage, {"float32": 0, "float16": 1, "bfloat16": 2})
        o.checkpoint_every = int(checkpoint_every)
        o.max_iterations = int(max_iterations)
        o.check_every = int(check_every)
        o.tolerance = float(tolerance)
        o.record_budget_bytes = int(record_budget_bytes)
        o.objective = _choice("objective", objective,
                              {"final": _abi.LBM_OBJ_FINAL, "time_average": _abi.LBM_OBJ_TIME_AVERAGE})
        o.checkpointing = _choice("checkpointing", checkpointing,
                                  {"every": _abi.LBM_CKPT_EVERY, "binomial": _abi.LBM_CKPT_BINOMIAL})
        o.snapshots = int(snapshots)
        grad = np.empty(self.shape)
        rep = _abi.AdjointReport()
        st = self.lib.lbm_gradient(self.h, _dp(w), C.byref(o), _dp(grad), C.byref(rep))
        report = AdjointReport(
            rep.residual,
            int(rep.iterations),
            int(rep.forward_recomputed),
            int(rep.peak_state_bytes),
            bool(rep.converged),
            rep.forward_ms,
            rep.adjoint_ms,
            rep.sensitivity_ms,
        )
        self.last_report = report
        self._check(st)
        return grad, report

    def step_vjp(self, state: np.ndarray, lambda_next: np.ndarray) -> tuple[np.ndarray, np.ndarray]:
        s = np.ascontiguousarray(state, dtype=np.float64).reshape(-1)
        ln = np.ascontiguousarray(lambda_next, dtype=np.float64).reshape(-1)
        lam = np.empty_like(s)
        ab = np.empty(self.cells)
        self._check(self.lib.lbm_step_vjp(self.h, _dp(s), _dp(ln), _dp(lam), _dp(ab), s.size))
        return lam.reshape(self.cells, self.q), ab

    def set_tau(self, tau: np.ndarray | None):
        """Per-cell relaxation times (Tau::PerCell, BGK problems), or None for
        the problem's uniform tau."""
        if tau is None:
            self._check(self.lib.lbm_set_tau(self.h, None, 0))
            return
        t = np.ascontiguousarray(tau, dtype=np.float64).reshape(-1)
        self._check(self.lib.lbm_set_tau(self.h, _dp(t), t.size))

    def step_vjp_tau(self, state: np.ndarray, lambda_next: np.ndarray):
        """step_vjp plus the per-cell cotangent of the relaxation time."""
        s = np.ascontiguousarray(state, dtype=np.float64).reshape(-1)
        ln = np.ascontiguousarray(lambda_next, dtype=np.float64).reshape(-1)
        lam = np.empty_like(s)
        ab, tb = np.empty(self.cells), np.empty(self.cells)
        self._check(self.lib.lbm_step_vjp_tau(self.h, _dp(s), _dp(ln), _dp(lam), _dp(ab), _dp(tb), s.size))
        return lam.reshape(self.cells, self.q), ab, tb

    def design_vjp(self, phi_bar: np.ndarray) -> np.ndarray:
        pb = np.ascontiguousarray(phi_bar, dtype=np.float64).reshape(-1)
        out = np.empty(self.cells)
        self._check(self.lib.lbm_design_vjp(self.h, _dp(pb), _dp(out), pb.size))
        return out.reshape(self.shape)
