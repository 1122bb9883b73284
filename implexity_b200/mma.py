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
        ("inner_iterations", C.c_int64),
        ("conservative", C.c_int32),
    ]


class GcmmaOptions(C.Structure):
    _fields_ = [
        ("rho_min", C.c_double),
        ("rho_init", C.c_double),
        ("rho_growth", C.c_double),
        ("max_conservative", C.c_int64),
    ]


# int eval_true(const double* x, double* f0, double* fs, void* ctx)
EVAL_FN = C.CFUNCTYPE(C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double), C.c_void_p)


EXPORTS = ["mma_default_options", "mma_create", "mma_destroy", "mma_last_error", "mma_step", "mma_kkt_residual",
           "mma_state", "mma_gcmma_default_options", "mma_enable_gcmma", "mma_step_gcmma", "mma_gcmma_state"]

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
    lib.mma_gcmma_default_options.argtypes = [C.POINTER(GcmmaOptions)]
    lib.mma_gcmma_default_options.restype = None
    lib.mma_enable_gcmma.argtypes = [C.c_void_p, C.POINTER(GcmmaOptions)]
    lib.mma_enable_gcmma.restype = C.c_int
    lib.mma_step_gcmma.argtypes = [C.c_void_p, dp, dp, dp, C.c_double, dp, dp, dp, EVAL_FN, C.c_void_p, dp,
                                   C.POINTER(Info)]
    lib.mma_step_gcmma.restype = C.c_int
    lib.mma_gcmma_state.argtypes = [C.c_void_p, dp, C.POINTER(C.c_int64)]
    lib.mma_gcmma_state.restype = C.c_int64
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
    inner_iterations: int = 0
    conservative: bool = True


def default_gcmma_options() -> dict:
    g = GcmmaOptions()
    load().mma_gcmma_default_options(C.byref(g))
    return {k: getattr(g, k) for k, _ in GcmmaOptions._fields_}


class MmaOptimizer:
    """MMA for min f0(x) s.t. f_j(x) <= 0 (j < m), x_min <= x <= x_max.

    ``gcmma`` (a dict of GcmmaOptions fields, or True for the defaults) makes
    it the reference's GCMMA optimiser (``MmaOptimizer::gcmma``): ``step``
    then refuses and ``step_gcmma`` runs the conservative inner loop."""

    def __init__(self, n: int, m: int, x_min=0.0, x_max=1.0, a=None, c=None, d=None, gcmma=None, **options):
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
        if gcmma is not None and gcmma is not False:
            g = GcmmaOptions()
            self.lib.mma_gcmma_default_options(C.byref(g))
            for k, v in (gcmma.items() if isinstance(gcmma, dict) else ()):
                if not hasattr(g, k):
                    raise ContractError(f"GCMMA: unknown option {k}")
                setattr(g, k, v)
            self._check(self.lib.mma_enable_gcmma(self.h, C.byref(g)), self.h)

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
        self.last = self._info(info)
        return out

    @staticmethod
    def _info(info) -> StepInfo:
        return StepInfo(info.iteration, info.kkt_residual, info.subproblem_kkt, bool(info.subproblem_converged),
                        info.subproblem_ip_residual, info.z, info.newton_steps, info.wallclock_s,
                        int(info.inner_iterations), bool(info.conservative))

    def step_gcmma(self, x_k, x_km1, x_km2, f0: float, df0dx, fs, dfsdx, eval_true) -> np.ndarray:
        """One GCMMA step; eval_true(x) -> (f0, fs) gives the true values at a
        trial point.  An exception raised by eval_true aborts the step and is
        re-raised here."""
        n, m = self.n, self.m
        xk, x1, x2, g0 = (_vec(v, n, name) for v, name in
                          ((x_k, "x_k"), (x_km1, "x_km1"), (x_km2, "x_km2"), (df0dx, "df0dx")))
        f = _vec(fs, m, "fs")
        df = _vec(dfsdx, m * n, "dfsdx")
        out = np.empty(n)
        info = Info()
        raised = []

        def cb(xp, f0p, fsp, _ctx):
            try:
                x = np.ctypeslib.as_array(xp, shape=(n,)).copy()
                v0, vs = eval_true(x)
                f0p[0] = float(v0)
                vs = np.asarray(vs, dtype=np.float64).ravel()
                if vs.size != m:
                    raise ContractError(f"GCMMA: eval_true returned {vs.size} constraint values, expected {m}")
                for j in range(m):
                    fsp[j] = float(vs[j])
                return 0
            except BaseException as e:  # noqa: BLE001  (re-raised after the C call returns)
                raised.append(e)
                return 1

        fn = EVAL_FN(cb)
        st = self.lib.mma_step_gcmma(self.h, _p(xk), _p(x1), _p(x2), float(f0), _p(g0), _p(f), _p(df), fn, None,
                                     _p(out), C.byref(info))
        if raised:
            raise raised[0]
        self._check(st, self.h)
        self.last = self._info(info)
        return out

    def gcmma_state(self) -> dict:
        rho = np.empty(self.m + 1)
        nf = C.c_int64()
        k = self.lib.mma_gcmma_state(self.h, _p(rho), C.byref(nf))
        return {"rho": rho[:max(k, 0)], "nonfinite_trials": int(nf.value)}

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
