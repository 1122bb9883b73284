"""ctypes mirror of include/lbm_b200.h and the loader of liblbm_b200.so.

The library is the product: there is no fallback.  ``load()`` raises if the
in-tree shared library is missing or was built for another ABI version.
"""
from __future__ import annotations

import ctypes as C
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "liblbm_b200.so"
ABI_VERSION = 6

# status codes
LBM_OK, LBM_E_CONTRACT, LBM_E_CONVERGENCE, LBM_E_CUDA, LBM_E_STATE = 0, 1, 2, 3, 4
STATUS_NAMES = {0: "OK", 1: "CONTRACT", 2: "CONVERGENCE", 3: "CUDA", 4: "STATE"}

LBM_BGK, LBM_TRT, LBM_MRT = 0, 1, 2
LBM_STORE_F32, LBM_STORE_F16, LBM_STORE_BF16 = 0, 1, 2
LBM_PORT_VELOCITY, LBM_PORT_PRESSURE = 0, 1
FACES = ["xmin", "xmax", "ymin", "ymax", "zmin", "zmax"]
LBM_FILTER_CONIC, LBM_FILTER_BOX = 0, 1
LBM_ADJ_HORIZON, LBM_ADJ_STEADY = 0, 1
LBM_OBJ_FINAL, LBM_OBJ_TIME_AVERAGE = 0, 1
LBM_CKPT_EVERY, LBM_CKPT_BINOMIAL = 0, 1
N_RESPONSES = 8
MAX_PORTS = 7

EXPORTS = [
    "lbm_create",
    "lbm_destroy",
    "lbm_last_error",
    "lbm_abi_version",
    "lbm_info",
    "lbm_set_design",
    "lbm_get_design",
    "lbm_forward",
    "lbm_set_populations",
    "lbm_get_populations",
    "lbm_advance",
    "lbm_trajectory",
    "lbm_responses",
    "lbm_time_average",
    "lbm_binomial_plan",
    "lbm_probe_bounded_wait",
    "lbm_wall_loads",
    "lbm_fields",
    "lbm_gradient",
    "lbm_step_vjp",
    "lbm_step_vjp_tau",
    "lbm_set_tau",
    "lbm_design_vjp",
    "lbm_create_slab",
    "lbm_slab_begin",
    "lbm_slab_step",
    "lbm_slab_inspect",
    "lbm_halo_bytes",
    "lbm_halo_pack",
    "lbm_halo_unpack",
    "lbm_slab_adjoint_begin",
    "lbm_slab_adjoint_step",
    "lbm_slab_gradient",
    "lbm_state_stats_noalloc",
]


class Port(C.Structure):
    _fields_ = [
        ("kind", C.c_int32),
        ("face", C.c_int32),
        ("mask", C.POINTER(C.c_uint8)),
        ("velocity_m_s", C.c_double * 3),
        ("gauge_pressure_Pa", C.c_double),
        ("amplitude_m_s", C.c_double * 3),
        ("amplitude_Pa", C.c_double),
        ("frequency_hz", C.c_double),
        ("phase_rad", C.c_double),
        ("ramp_s", C.c_double),
        ("reconstruction", C.c_int32),
    ]


class Problem(C.Structure):
    _fields_ = [
        ("lattice", C.c_int32),
        ("collision", C.c_int32),
        ("storage", C.c_int32),
        ("shape", C.c_int32 * 3),
        ("periodic_axes", C.c_int32 * 3),
        ("n_ports", C.c_int32),
        ("step_count", C.c_int64),
        ("spacing_m", C.c_double),
        ("step_s", C.c_double),
        ("density_kg_m3", C.c_double),
        ("kinematic_viscosity_m2_s", C.c_double),
        ("acceleration_m_s2", C.c_double * 3),
        ("drag_max_per_s", C.c_double),
        ("drag_shape", C.c_double),
        ("mach_limit", C.c_double),
        ("filter_radius_m", C.c_double),
        ("projection_beta", C.c_double),
        ("projection_eta", C.c_double),
        ("filter_kind", C.c_int32),
        ("box_half_width", C.c_int32),
        ("trt_magic", C.c_double),
        ("mrt_odd_magic", C.c_double),
        ("mrt_bulk_rate", C.c_double),
        ("mrt_even_rate", C.c_double),
        ("solid_mask", C.POINTER(C.c_uint8)),
        ("design_region", C.POINTER(C.c_uint8)),
        ("fixed_design", C.POINTER(C.c_double)),
        ("ports", C.POINTER(Port)),
        ("time_average", C.c_int32),
        ("collision_fp64", C.c_int32),
    ]


class Diag(C.Structure):
    _fields_ = [
        ("maximum_mach", C.c_double),
        ("relative_mass_drift", C.c_double),
        ("relaxation_time", C.c_double),
        ("minimum_population", C.c_double),
        ("boundary_exchange_total", C.c_double),
        ("steps", C.c_int64),
        ("nonfinite", C.c_int32),
        ("admitted", C.c_int32),
        ("device_ms", C.c_double),
    ]


class AdjointOpts(C.Structure):
    _fields_ = [
        ("mode", C.c_int32),
        ("lambda_storage", C.c_int32),
        ("checkpoint_every", C.c_int64),
        ("max_iterations", C.c_int64),
        ("check_every", C.c_int64),
        ("tolerance", C.c_double),
        ("record_budget_bytes", C.c_int64),
        ("objective", C.c_int32),
        ("checkpointing", C.c_int32),
        ("snapshots", C.c_int64),
    ]


class SlabDiag(C.Structure):
    _fields_ = [
        ("mass", C.c_double),
        ("exchange", C.c_double),
        ("minimum_population", C.c_double),
        ("maximum_speed2", C.c_double),
        ("nonfinite", C.c_int32),
    ]


class AdjointReport(C.Structure):
    _fields_ = [
        ("residual", C.c_double),
        ("iterations", C.c_int64),
        ("forward_recomputed", C.c_int64),
        ("peak_state_bytes", C.c_int64),
        ("converged", C.c_int32),
        ("forward_ms", C.c_double),
        ("adjoint_ms", C.c_double),
        ("sensitivity_ms", C.c_double),
    ]


class Info(C.Structure):
    _fields_ = [
        ("cells", C.c_int64),
        ("fluid_cells", C.c_int64),
        ("q", C.c_int32),
        ("n_ports", C.c_int32),
        ("tau", C.c_double),
        ("acceleration_lattice", C.c_double * 3),
        ("device_bytes", C.c_int64),
    ]


_dp = C.POINTER(C.c_double)
_lib = None


def _declare(lib: C.CDLL) -> None:
    h = C.c_void_p
    lib.lbm_create.argtypes = [C.POINTER(Problem), C.POINTER(C.c_void_p)]
    lib.lbm_destroy.argtypes = [h]
    lib.lbm_destroy.restype = None
    lib.lbm_last_error.argtypes = [h]
    lib.lbm_last_error.restype = C.c_char_p
    lib.lbm_abi_version.argtypes = []
    lib.lbm_info.argtypes = [h, C.POINTER(Info)]
    lib.lbm_set_design.argtypes = [h, _dp, C.c_size_t]
    lib.lbm_get_design.argtypes = [h, _dp, _dp]
    lib.lbm_forward.argtypes = [h, C.c_int64, C.POINTER(Diag)]
    lib.lbm_set_populations.argtypes = [h, _dp, C.c_size_t]
    lib.lbm_get_populations.argtypes = [h, _dp, C.c_size_t]
    lib.lbm_advance.argtypes = [h, C.c_int64, C.POINTER(Diag)]
    lib.lbm_trajectory.argtypes = [h, _dp, _dp, _dp, _dp, C.c_size_t]
    lib.lbm_responses.argtypes = [h, _dp]
    lib.lbm_time_average.argtypes = [h, _dp]
    lib.lbm_binomial_plan.argtypes = [C.c_int64, C.c_int64, C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
    lib.lbm_probe_bounded_wait.argtypes = [C.c_int64, C.POINTER(C.c_int32), C.POINTER(C.c_double)]
    lib.lbm_wall_loads.argtypes = [h, C.c_double, _dp, _dp, _dp, C.c_size_t, C.POINTER(C.c_size_t)]
    lib.lbm_fields.argtypes = [h, _dp, _dp, _dp]
    lib.lbm_gradient.argtypes = [h, _dp, C.POINTER(AdjointOpts), _dp, C.POINTER(AdjointReport)]
    lib.lbm_step_vjp.argtypes = [h, _dp, _dp, _dp, _dp, C.c_size_t]
    lib.lbm_create_slab.argtypes = [C.POINTER(Problem), C.c_int32, C.c_int32, C.c_int32, C.POINTER(h)]
    lib.lbm_slab_begin.argtypes = [h]
    lib.lbm_slab_step.argtypes = [h, C.POINTER(SlabDiag)]
    lib.lbm_slab_inspect.argtypes = [h, C.POINTER(SlabDiag)]
    lib.lbm_halo_bytes.argtypes = [h, C.c_int32, C.POINTER(C.c_size_t)]
    lib.lbm_halo_pack.argtypes = [h, C.c_int32, C.c_int32, C.c_void_p]
    lib.lbm_halo_unpack.argtypes = [h, C.c_int32, C.c_int32, C.c_void_p]
    lib.lbm_slab_adjoint_begin.argtypes = [h, _dp, _dp]
    lib.lbm_slab_adjoint_step.argtypes = [h, _dp]
    lib.lbm_slab_gradient.argtypes = [h, _dp, C.c_size_t]
    lib.lbm_step_vjp_tau.argtypes = [h, _dp, _dp, _dp, _dp, _dp, C.c_size_t]
    lib.lbm_set_tau.argtypes = [h, _dp, C.c_size_t]
    lib.lbm_design_vjp.argtypes = [h, _dp, _dp, C.c_size_t]
    lib.lbm_state_stats_noalloc.argtypes = [C.c_int32, C.c_int64, C.c_void_p, C.c_void_p, C.c_void_p, _dp,
                                            C.c_void_p, C.c_void_p]
    for name in EXPORTS:
        fn = getattr(lib, name)
        if name not in ("lbm_destroy", "lbm_last_error"):
            fn.restype = C.c_int32


def load(path: Path | str | None = None) -> C.CDLL:
    """Loads liblbm_b200.so (once) and checks its ABI version."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build it with `python -m implexity_b200.build` (the CUDA library has no fallback)"
        )
    lib = C.CDLL(str(p))
    _declare(lib)
    v = lib.lbm_abi_version()
    if v != ABI_VERSION:
        raise RuntimeError(f"{p} has ABI version {v}, expected {ABI_VERSION}")
    if path is None:
        _lib = lib
    return lib
