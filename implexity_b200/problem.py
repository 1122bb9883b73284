"""JSON problem mapping -> lbm_problem_t, mirroring LbmProblem::normalize.

The reference parses the problem with serde (crates/implexity-physics-lbm/src/
solver.rs:414-550): exact key set, array shapes and dtypes.  Those structural
checks live here with the reference's messages; the numeric checks (positive
scalars, relaxation time, ports, topology map) are applied by lbm_create in the
CUDA library, also with the reference's messages.

One optional key is added to the reference's OPTIONAL_KEYS: ``solver_options``
selects the lattice (D3Q19/D3Q27), the collision operator (bgk/trt/mrt with
their parameters, moving/collision.rs:38-53), the population storage
(float32/float16/bfloat16), a box design filter, and the adjoint mode.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass, field
from typing import Any

import numpy as np

from . import _abi

PROBLEM_KEYS = sorted(
    [
        "acceleration_m_s2",
        "density_kg_m3",
        "design_region",
        "drag_max_per_s",
        "drag_shape",
        "fixed_design",
        "history_byte_budget",
        "kinematic_viscosity_m2_s",
        "mach_limit",
        "periodic_axes",
        "shape",
        "solid_mask",
        "spacing_m",
        "step_count",
        "step_s",
    ]
)
# port reconstructions (ports.rs:134-147) and the moving engine's extrapolation (moving/boundary.rs:445-506)
RECONSTRUCTIONS = {
    "legacy_moment": 0,
    "neighbor_non_equilibrium": 1,
    "non_equilibrium_extrapolation": 2,
    "regularized_known_stress": 3,
}
OPTIONAL_KEYS = ["topology_map", "ports", "origin_m", "field_registration", "geometry_source", "solver_options"]

STORAGE = {"float32": _abi.LBM_STORE_F32, "float16": _abi.LBM_STORE_F16, "bfloat16": _abi.LBM_STORE_BF16}
COLLISIONS = {"bgk": _abi.LBM_BGK, "trt": _abi.LBM_TRT, "mrt": _abi.LBM_MRT}


class ContractError(ValueError):
    """CaeError::Contract (implexity-core/src/error.rs:34-56)."""


def _err(msg: str) -> ContractError:
    return ContractError(msg)


def _scalar(v: Any) -> float | None:
    try:
        a = np.asarray(v, dtype=float)
    except (TypeError, ValueError):
        return None
    if a.shape != () or isinstance(v, bool) or not math.isfinite(float(a)):
        return None
    return float(a)


def _int(v: Any) -> int | None:
    if isinstance(v, bool):
        return None
    if isinstance(v, (int, np.integer)):
        return int(v)
    if isinstance(v, float) and v.is_integer():
        return int(v)
    return None


def _bool_array(v: Any, shape: tuple[int, ...]) -> np.ndarray | None:
    try:
        a = np.asarray(v)
    except (TypeError, ValueError):
        return None
    if a.shape != shape or a.dtype != np.bool_:
        return None
    return np.ascontiguousarray(a, dtype=np.uint8)


@dataclass
class SolverOptions:
    lattice: int = 19
    collision: str = "bgk"
    trt_magic: float = 3.0 / 16.0
    mrt_odd_magic: float = 3.0 / 16.0
    mrt_bulk_rate: float | None = None
    mrt_even_rate: float | None = None
    storage: str = "float32"
    box_half_width: int = 0
    adjoint: str = "horizon"          # "horizon" (reference) or "steady"
    lambda_storage: str = "float32"
    checkpoint_every: int = 0
    tolerance: float = 1e-8
    max_iterations: int = 100000
    time_average: bool = False        # also evaluate the responses of every state (stage objective)
    collision_arithmetic: str = "float32"  # "float64": FP64 collision on FP32 storage

    @classmethod
    def parse(cls, v: Any) -> "SolverOptions":
        o = cls()
        if v is None:
            return o
        if not isinstance(v, dict):
            raise _err("solver_options must be a mapping")
        known = {"lattice", "collision", "population_storage", "filter", "adjoint", "time_average",
                 "collision_arithmetic"}
        if set(v) - known:
            raise _err("solver_options accepts lattice, collision, population_storage, filter, adjoint, "
                       "time_average and collision_arithmetic")
        ca = v.get("collision_arithmetic", "float32")
        if ca not in ("float32", "float64"):
            raise _err("solver_options.collision_arithmetic must be float32 or float64")
        o.collision_arithmetic = ca
        ta = v.get("time_average", False)
        if not isinstance(ta, bool):
            raise _err("solver_options.time_average must be a boolean")
        o.time_average = ta
        lat = v.get("lattice", "D3Q19")
        if lat not in ("D3Q19", "D3Q27"):
            raise _err("solver_options.lattice must be D3Q19 or D3Q27")
        o.lattice = int(lat[3:])
        col = v.get("collision", {"kind": "bgk"})
        if isinstance(col, str):
            col = {"kind": col}
        kind = col.get("kind") if isinstance(col, dict) else None
        if kind not in COLLISIONS:
            raise _err("collision kind must be bgk, trt or mrt")
        o.collision = kind
        if kind == "trt":
            o.trt_magic = float(col.get("magic", 3.0 / 16.0))
        if kind == "mrt":
            o.mrt_odd_magic = float(col.get("odd_magic", 3.0 / 16.0))
            b, e = col.get("bulk_rate"), col.get("even_rate")
            o.mrt_bulk_rate = None if b is None else float(b)
            o.mrt_even_rate = None if e is None else float(e)
        st = v.get("population_storage", "float32")
        if st not in STORAGE:
            raise _err("population_storage must be float32, float16 or bfloat16")
        o.storage = st
        flt = v.get("filter")
        if flt is not None:
            if not isinstance(flt, dict) or flt.get("kind") != "box" or _int(flt.get("half_width")) is None:
                raise _err("filter must be {'kind': 'box', 'half_width': int}")
            o.box_half_width = int(flt["half_width"])
        adj = v.get("adjoint")
        if adj is not None:
            if not isinstance(adj, dict) or adj.get("mode", "horizon") not in ("horizon", "steady"):
                raise _err("adjoint.mode must be horizon or steady")
            o.adjoint = adj.get("mode", "horizon")
            ls = adj.get("lambda_storage", "float32")
            if ls not in STORAGE:
                raise _err("adjoint.lambda_storage must be float32, float16 or bfloat16")
            o.lambda_storage = ls
            o.checkpoint_every = int(adj.get("checkpoint_every", 0))
            o.tolerance = float(adj.get("tolerance", 1e-8))
            o.max_iterations = int(adj.get("max_iterations", 100000))
        return o


@dataclass
class NormalizedProblem:
    """Host arrays kept alive for the lbm_problem_t that points into them."""

    shape: tuple[int, int, int]
    spacing_m: float
    step_s: float
    step_count: int
    density_kg_m3: float
    kinematic_viscosity_m2_s: float
    acceleration_m_s2: tuple[float, float, float]
    periodic_axes: tuple[bool, bool, bool]
    solid_mask: np.ndarray
    design_region: np.ndarray
    fixed_design: np.ndarray
    drag_max_per_s: float
    drag_shape: float
    mach_limit: float
    history_byte_budget: int
    topology_map: dict
    ports: list[dict]
    options: SolverOptions
    origin_m: tuple[float, float, float] = (0.0, 0.0, 0.0)
    _keep: list = field(default_factory=list, repr=False)

    @property
    def cells(self) -> int:
        return int(np.prod(self.shape))

    @property
    def tau(self) -> float:
        return 0.5 + 3.0 * self.kinematic_viscosity_m2_s * self.step_s / (self.spacing_m**2)

    def to_c(self) -> _abi.Problem:
        p = _abi.Problem()
        o = self.options
        p.lattice = o.lattice
        p.collision = COLLISIONS[o.collision]
        p.storage = STORAGE[o.storage]
        for a in range(3):
            p.shape[a] = self.shape[a]
            p.periodic_axes[a] = 1 if self.periodic_axes[a] else 0
            p.acceleration_m_s2[a] = self.acceleration_m_s2[a]
        p.step_count = self.step_count
        p.spacing_m = self.spacing_m
        p.step_s = self.step_s
        p.density_kg_m3 = self.density_kg_m3
        p.kinematic_viscosity_m2_s = self.kinematic_viscosity_m2_s
        p.drag_max_per_s = self.drag_max_per_s
        p.drag_shape = self.drag_shape
        p.mach_limit = self.mach_limit
        tm = self.topology_map
        p.filter_radius_m = tm["filter_radius_m"]
        p.projection_beta = tm["projection_beta"]
        p.projection_eta = tm["projection_eta"]
        p.filter_kind = _abi.LBM_FILTER_BOX if o.box_half_width > 0 else _abi.LBM_FILTER_CONIC
        p.box_half_width = o.box_half_width
        nan = float("nan")
        p.trt_magic = o.trt_magic
        p.mrt_odd_magic = o.mrt_odd_magic
        p.mrt_bulk_rate = nan if o.mrt_bulk_rate is None else o.mrt_bulk_rate
        p.mrt_even_rate = nan if o.mrt_even_rate is None else o.mrt_even_rate
        p.solid_mask = self.solid_mask.ctypes.data_as(C.POINTER(C.c_uint8))
        p.design_region = self.design_region.ctypes.data_as(C.POINTER(C.c_uint8))
        p.fixed_design = self.fixed_design.ctypes.data_as(C.POINTER(C.c_double))
        ports = (_abi.Port * max(1, len(self.ports)))()
        for k, port in enumerate(self.ports):
            ports[k].kind = _abi.LBM_PORT_PRESSURE if port["kind"] == "pressure" else _abi.LBM_PORT_VELOCITY
            ports[k].face = _abi.FACES.index(port["face"])
            ports[k].mask = port["mask"].ctypes.data_as(C.POINTER(C.c_uint8))
            for a in range(3):
                ports[k].velocity_m_s[a] = port["velocity_m_s"][a]
            ports[k].gauge_pressure_Pa = port.get("gauge_pressure_Pa", 0.0)
            for a in range(3):
                ports[k].amplitude_m_s[a] = port.get("amplitude_m_s", [0.0, 0.0, 0.0])[a]
            ports[k].amplitude_Pa = port.get("amplitude_Pa", 0.0)
            ports[k].frequency_hz = port.get("frequency_hz", 0.0)
            ports[k].phase_rad = port.get("phase_rad", 0.0)
            ports[k].ramp_s = port.get("ramp_s", 0.0)
            ports[k].reconstruction = RECONSTRUCTIONS[port.get("reconstruction", "legacy_moment")]
        p.n_ports = len(self.ports)
        p.time_average = 1 if o.time_average else 0
        p.collision_fp64 = 1 if o.collision_arithmetic == "float64" else 0
        p.ports = C.cast(ports, C.POINTER(_abi.Port))
        self._keep = [ports, p]
        return p


def _ports(value: Any, shape: tuple[int, int, int]) -> list[dict]:
    """Structural half of normalize_ports (ports.rs:106-160)."""
    if not isinstance(value, list):
        raise _err("ports must be a list")
    out, ids = [], set()
    for port in value:
        kind = port.get("kind") if isinstance(port, dict) else None
        if kind not in ("velocity", "pressure"):
            raise _err("Port kind must be velocity or pressure")
        required = {"id", "kind", "face", "mask", "velocity_m_s"} | ({"gauge_pressure_Pa"} if kind == "pressure" else set())
        # pulsatile signal (moving/boundary.rs Signal; keys of implexity-physics-fsi problem/fluid.rs:256-322)
        signal_keys = {"frequency_hz", "phase_rad", "ramp_s"} | (
            {"amplitude_Pa"} if kind == "pressure" else {"amplitude_m_s"})
        keys = set(port) - {"reconstruction"} - signal_keys
        pid = port.get("id")
        if keys != required or not isinstance(pid, str) or not pid.strip() or pid in ids:
            raise _err("Unique port id and exact port fields required")
        rec = port.get("reconstruction", "legacy_moment")
        if rec not in ("legacy_moment", "regularized_known_stress", "neighbor_non_equilibrium",
                       "non_equilibrium_extrapolation"):
            raise _err(
                "Port reconstruction must be legacy_moment, regularized_known_stress or neighbor_non_equilibrium"
            )
        ids.add(pid)
        if port.get("face") not in _abi.FACES:
            raise _err("Port must identify one Cartesian face")
        mask = _bool_array(port.get("mask"), shape)
        if mask is None or not mask.any():
            raise _err("Nonempty shape-matched boolean port mask required")
        vel = np.asarray(port.get("velocity_m_s"), dtype=float) if port.get("velocity_m_s") is not None else None
        if vel is None or vel.shape != (3,) or not np.all(np.isfinite(vel)):
            raise _err("Port velocity requires three finite components")
        entry = {"id": pid, "kind": kind, "face": port["face"], "mask": mask, "velocity_m_s": [float(x) for x in vel],
                 "reconstruction": rec}
        if kind == "pressure":
            g = _scalar(port.get("gauge_pressure_Pa"))
            if g is None:
                raise _err("Finite scalar gauge pressure required")
            entry["gauge_pressure_Pa"] = g
        for key, lo in (("frequency_hz", 0.0), ("phase_rad", None), ("ramp_s", 0.0)):
            if key in port:
                val = _scalar(port[key])
                if val is None or (lo is not None and val < lo):
                    raise _err(f"Port {key} must be a finite" + (" nonnegative" if lo is not None else "") + " scalar")
                entry[key] = val
        if kind == "velocity" and "amplitude_m_s" in port:
            amp = np.asarray(port["amplitude_m_s"], dtype=float)
            if amp.shape != (3,) or not np.all(np.isfinite(amp)):
                raise _err("Port amplitude_m_s requires three finite components")
            entry["amplitude_m_s"] = [float(x) for x in amp]
        if kind == "pressure" and "amplitude_Pa" in port:
            amp_p = _scalar(port["amplitude_Pa"])
            if amp_p is None:
                raise _err("Port amplitude_Pa must be a finite scalar")
            entry["amplitude_Pa"] = amp_p
        out.append(entry)
    return out


def normalize(problem: Any) -> NormalizedProblem:
    """Structural normalisation of the problem mapping (solver.rs:414-470)."""
    keys_ok = isinstance(problem, dict) and sorted(k for k in problem if k not in OPTIONAL_KEYS) == PROBLEM_KEYS
    if not keys_ok:
        lst = ", ".join(f"'{k}'" for k in PROBLEM_KEYS)
        raise _err(f"LBM requires exactly these problem keys: [{lst}]")
    p = problem
    shp = p["shape"]
    if not isinstance(shp, (list, tuple)) or len(shp) != 3 or any(_int(v) is None or _int(v) < 2 for v in shp):
        raise _err("LBM shape must contain three integers >= 2")
    shape = tuple(int(v) for v in shp)
    vals = {}
    for key in ("spacing_m", "step_s", "density_kg_m3", "kinematic_viscosity_m2_s", "drag_max_per_s", "drag_shape", "mach_limit"):
        v = _scalar(p[key])
        if v is None or v <= 0:
            raise _err(f"{key} must be a finite positive scalar")
        vals[key] = v
    if vals["mach_limit"] > 0.2:
        raise _err("LBM mach_limit must be <= 0.2; this is not a compressible gas solver")
    count = _int(p["step_count"])
    if count is None or not (1 <= count <= 1_000_000):
        raise _err("step_count must be an integer in [1,1000000]")
    cells = shape[0] * shape[1] * shape[2]
    required = (count + 1) * cells * 19 * 8
    budget = _int(p["history_byte_budget"])
    if budget is None or budget < required:
        raise _err("Population history exceeds explicit byte budget; AD working memory is additional")
    if "geometry_source" in p or "field_registration" in p:
        raise _err("geometry_source and field_registration are not provided by the GPU provider")
    masks = []
    for key in ("solid_mask", "design_region"):
        a = _bool_array(p[key], shape)
        if a is None:
            raise _err(f"{key} must be a shape-matched boolean array")
        masks.append(a)
    try:
        fixed = np.asarray(p["fixed_design"])
    except (TypeError, ValueError):
        fixed = None
    if (
        fixed is None
        or fixed.shape != shape
        or not (np.issubdtype(fixed.dtype, np.floating) or np.issubdtype(fixed.dtype, np.integer))
        or fixed.dtype == np.bool_
        or not np.all(np.isfinite(fixed))
        or np.any((fixed < 0) | (fixed > 1))
    ):
        raise _err("fixed_design must be finite and in [0,1]")
    solid, design = masks
    if solid.all() or np.any(solid.astype(bool) & design.astype(bool)):
        raise _err("Need fluid cells; fixed solid cells cannot be designable")
    acc = np.asarray(p["acceleration_m_s2"], dtype=float) if p["acceleration_m_s2"] is not None else None
    if acc is None or acc.shape != (3,) or not np.all(np.isfinite(acc)):
        raise _err("acceleration_m_s2 requires three finite components")
    per = p["periodic_axes"]
    if not isinstance(per, (list, tuple)) or len(per) != 3 or not all(isinstance(v, bool) for v in per):
        raise _err("periodic_axes requires three booleans; false means closed no-slip walls")
    tm = p.get("topology_map", {"filter_radius_m": 0.0, "projection_beta": 0.0, "projection_eta": 0.5})
    if not isinstance(tm, dict) or sorted(tm) != ["filter_radius_m", "projection_beta", "projection_eta"]:
        raise _err("topology_map requires filter_radius_m, projection_beta and projection_eta")
    topo = {}
    for k, v in tm.items():
        s = _scalar(v)
        if s is None:
            raise _err(f"topology_map.{k} must be finite real scalar")
        topo[k] = s
    ports = _ports(p.get("ports", []), shape)
    origin = p.get("origin_m", [0.0, 0.0, 0.0])
    opts = SolverOptions.parse(p.get("solver_options"))
    return NormalizedProblem(
        shape=shape,
        spacing_m=vals["spacing_m"],
        step_s=vals["step_s"],
        step_count=count,
        density_kg_m3=vals["density_kg_m3"],
        kinematic_viscosity_m2_s=vals["kinematic_viscosity_m2_s"],
        acceleration_m_s2=tuple(float(x) for x in acc),
        periodic_axes=tuple(per),
        solid_mask=solid,
        design_region=design,
        fixed_design=np.ascontiguousarray(fixed, dtype=np.float64),
        drag_max_per_s=vals["drag_max_per_s"],
        drag_shape=vals["drag_shape"],
        mach_limit=vals["mach_limit"],
        history_byte_budget=budget,
        topology_map=topo,
        ports=ports,
        options=opts,
        origin_m=tuple(float(x) for x in origin),
    )
