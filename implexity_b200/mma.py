"""ctypes handle over the host MMA library (include/mma_cpu.h).

``MmaOptimizer`` mirrors the reference optimiser's interface
(crates/implexity-optim/src/mma.rs: ``MmaOptimizer::new``, ``step``,
``kkt_residual``, ``converged``, ``dual_variables``, ``state_dict``) on the
host CPU; the GPU never sees the design update.  Options default to the
reference's ``MmaOptions::default`` (mma.rs:107-129).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass
from pathlib import Path

import numpy as np

from .problem import ContractError

LIB_PATH = Path(__file__).resolve().parent / "libmma_cpu.so"

MMA_OK, MMA_E_CONTRACT, MMA_E_RUNTIME = 0, 1, 2


class Options(C.Structure):
    _fields_ = [
        ("move_limit", C.c_double),
        ("asymptote_init", C.c_double),
        ("asymptote_expand", C.c_double),
        ("asymptote_contract", C.c_double),
        ("asymptote_lo", C.c_double),
        ("asymptote_hi", C.c_double),
        ("a0", C.c_double),
        ("raa0", C.c_double),
        ("albefa", C.c_double),
        ("epsimin", C.c_double),
        ("max_inner", C.c_int64),
        ("strict_subproblem", C.c_int32),
    ]


class Info(C.Structure):
    _fields_ = [
        ("iteration", C.c_int64),
        ("kkt_residual", C.c_double),
        ("subproblem_kkt", C.c_double),
        ("subproblem_converged", C.c_int32),
        ("subproblem_ip_residual", C.c_double),
        ("z", C.c_double),
        ("newton_steps", C.c_int64),
        ("wallclock_s", C.c_double),
    ]


EXPORTS = ["mma_default_options", "mma_create", "mma_destroy", "mma_last_error", "mma_step", "mma_kkt_residual",
           "mma_state"]

_lib = None


def load(path: Path | str | None = None) -> C.CDLL:
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(f"{p} is missing: build it with `python -m implexity_b200.build`")
    lib = C.CDLL(str(p))
    dp = C.POINTER(C.c_double)
    lib.mma_default_options.argtypes = [C.POINTER(Options)]
    lib.mma_default_options.restype = None
    lib.mma_create.argtypes = [C.c_int64, C.c_int64, C.POINTER(Options), dp, dp, dp, dp, dp, C.c_int64,
                               C.POINTER(C.c_void_p)]
    lib.mma_create.restype = C.c_int
    lib.mma_destroy.argtypes = [C.c_void_p]
    lib.mma_destroy.restype = None
    lib.mma_last_error.argtypes = [C.c_void_p]
    lib.mma_last_error.restype = C.c_char_p
    lib.mma_step.argtypes = [C.c_void_p, dp, dp, dp, C.c_double, dp, dp, dp, dp, C.POINTER(Info)]
    lib.mma_step.restype = C.c_int
    lib.mma_kkt_residual.argtypes = [C.c_void_p, dp, dp, dp, dp]
    lib.mma_kkt_residual.restype = C.c_double
    lib.mma_state.argtypes = [C.c_void_p, dp, dp, dp, dp, dp]
    lib.mma_state.restype = C.c_int64
    if path is None:
        _lib = lib
    return lib


def _p(a: np.ndarray | None):
    return None if a is None else a.ctypes.data_as(C.POINTER(C.c_double))


def _vec(a, n: int, name: str) -> np.ndarray:
    v = np.ascontiguousarray(np.asarray(a, dtype=np.float64).ravel())
    if v.size != n:
        raise ContractError(f"MMA: {name} must have {n} entries")
    return v


def default_options() -> dict:
    o = Options()
    load().mma_default_options(C.byref(o))
    return {k: getattr(o, k) for k, _ in Options._fields_}


@dataclass
class StepInfo:
    iteration: int
    kkt_residual: float
    subproblem_kkt: float
    subproblem_converged: bool
    subproblem_ip_residual: float
    z: float
    newton_steps: int
    wallclock_s: float


class MmaOptimizer:
    """MMA for min f0(x) s.t. f_j(x) <= 0 (j < m), x_min <= x <= x_max."""

    def __init__(self, n: int, m: int, x_min=0.0, x_max=1.0, a=None, c=None, d=None, **options):
        self.lib = load()
        self.n, self.m = int(n), int(m)
        o = Options()
        self.lib.mma_default_options(C.byref(o))
        for k, v in options.items():
            if not hasattr(o, k):
                raise ContractError(f"MMA: unknown option {k}")
            setattr(o, k, v)
        lo = np.ascontiguousarray(np.atleast_1d(np.asarray(x_min, np.float64)).ravel())
        hi = np.ascontiguousarray(np.atleast_1d(np.asarray(x_max, np.float64)).ravel())
        if lo.size != hi.size:
            raise ContractError("MMA: x_min and x_max must have the same size")
        coef = [None if v is None else np.ascontiguousarray(np.broadcast_to(np.asarray(v, np.float64), (self.m,)))
                for v in (a, c, d)]
        self._keep = (lo, hi, coef)
        h = C.c_void_p()
        st = self.lib.mma_create(self.n, self.m, C.byref(o), *(_p(v) for v in coef), _p(lo), _p(hi), lo.size,
                                 C.byref(h))
        self._check(st, None)
        self.h = h
        self.last: StepInfo | None = None

    def _check(self, st: int, h):
        if st == MMA_OK:
            return
        msg = self.lib.mma_last_error(h).decode()
        if st == MMA_E_CONTRACT:
            raise ContractError(msg)
        raise RuntimeError(msg)

    def close(self):
        if getattr(self, "h", None):
            self.lib.mma_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def step(self, x_k, x_km1, x_km2, f0: float, df0dx, fs=None, dfsdx=None) -> np.ndarray:
        n, m = self.n, self.m
        xk, x1, x2, g0 = (_vec(v, n, name) for v, name in
                          ((x_k, "x_k"), (x_km1, "x_km1"), (x_km2, "x_km2"), (df0dx, "df0dx")))
        f = _vec(fs if fs is not None else [], m, "fs")
        df = _vec(dfsdx if dfsdx is not None else np.zeros((0,)), m * n, "dfsdx")
        out = np.empty(n)
        info = Info()
        st = self.lib.mma_step(self.h, _p(xk), _p(x1), _p(x2), float(f0), _p(g0), _p(f), _p(df), _p(out),
                               C.byref(info))
        self._check(st, self.h)
        self.last = StepInfo(info.iteration, info.kkt_residual, info.subproblem_kkt, bool(info.subproblem_converged),
                             info.subproblem_ip_residual, info.z, info.newton_steps, info.wallclock_s)
        return out

    def kkt_residual(self, x, df0dx, fs=None, dfsdx=None) -> float:
        n, m = self.n, self.m
        f = _vec(fs if fs is not None else [], m, "fs")
        df = _vec(dfsdx if dfsdx is not None else np.zeros((0,)), m * n, "dfsdx")
        return float(self.lib.mma_kkt_residual(self.h, _p(_vec(x, n, "x")), _p(_vec(df0dx, n, "df0dx")), _p(f),
                                               _p(df)))

    def converged(self, tol: float) -> bool:
        return self.last is not None and self.last.kkt_residual < tol

    def state_dict(self) -> dict:
        lam, y, z = np.empty(self.m), np.empty(self.m), np.empty(1)
        low, upp = np.full(self.n, np.nan), np.full(self.n, np.nan)
        it = self.lib.mma_state(self.h, _p(lam), _p(y), _p(z), _p(low), _p(upp))
        return {"l": low, "u": upp, "iter": int(it), "lam": lam, "y": y, "z": float(z[0])}

    def dual_variables(self) -> np.ndarray:
        return self.state_dict()["lam"]
