"""ctypes wrapper of the FP64 CPU oracle (oracle/liblbm_oracle.so).

TEST INFRASTRUCTURE ONLY.  Imported by tests/, by ``__graft_entry__.smoke()``
and by the ``cpu_baseline`` / ``--impl reference`` legs of bench.py, and only
as the checker or the timed CPU baseline.  Parity unpinned: see
oracle/lbm_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liblbm_oracle.so"

_dp = C.POINTER(C.c_double)


class Diag(C.Structure):
    _fields_ = [
        ("maximum_mach", C.c_double),
        ("relative_mass_drift", C.c_double),
        ("minimum_population", C.c_double),
        ("boundary_exchange_total", C.c_double),
        ("nonfinite", C.c_int32),
        ("admitted", C.c_int32),
    ]


class GradReport(C.Structure):
    _fields_ = [("iterations", C.c_int64), ("forward_evaluations", C.c_int64), ("residual", C.c_double)]


_lib = None


def build() -> Path:
    srcs = [HERE / "lbm_oracle.cpp", HERE / "lbm_oracle.h", HERE.parent / "include" / "lbm_b200.h"]
    if not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in srcs):
        subprocess.run(["make", "-s", "-C", str(HERE)], check=True)
    return LIB


def lib() -> C.CDLL:
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(str(LIB))
        h = C.c_void_p
        L.orc_create.argtypes = [C.c_void_p, C.POINTER(C.c_void_p)]
        L.orc_destroy.argtypes = [h]
        L.orc_destroy.restype = None
        L.orc_error.restype = C.c_char_p
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_set_threads.restype = None
        L.orc_info.argtypes = [h, C.POINTER(C.c_int64), C.POINTER(C.c_int32), _dp, _dp, C.POINTER(C.c_int64)]
        L.orc_info.restype = None
        for name in ("orc_design",):
            getattr(L, name).argtypes = [h, _dp, _dp, _dp]
            getattr(L, name).restype = None
        L.orc_design_vjp.argtypes = [h, _dp, _dp, _dp]
        L.orc_design_vjp.restype = None
        L.orc_resistance_derivative.argtypes = [h, _dp, _dp]
        L.orc_resistance_derivative.restype = None
        L.orc_initial.argtypes = [h, _dp]
        L.orc_initial.restype = None
        L.orc_interval.argtypes = [h, _dp, _dp, _dp]
        L.orc_interval.restype = C.c_double
        L.orc_history.argtypes = [h, _dp, C.c_int64, _dp, C.POINTER(Diag)]
        L.orc_history.restype = None
        L.orc_history_trace.argtypes = [h, _dp, C.c_int64, _dp, C.POINTER(Diag), _dp, _dp]
        L.orc_history_trace.restype = None
        L.orc_vector.argtypes = [h, _dp, _dp, _dp, _dp]
        L.orc_vector.restype = None
        L.orc_vector_vjp.argtypes = [h, _dp, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_vector_vjp.restype = None
        L.orc_interval_vjp.argtypes = [h, _dp, _dp, _dp, _dp, _dp]
        L.orc_interval_vjp.restype = None
        L.orc_gradient.argtypes = [h, _dp, _dp, C.c_int64, C.c_int, C.c_int64, C.c_double, C.c_int64, _dp, _dp,
                                   C.POINTER(GradReport)]
        L.orc_mrt_basis.argtypes = [C.c_int, _dp, _dp, C.POINTER(C.c_int32)]
        L.orc_set_tau.argtypes = [h, _dp]
        L.orc_set_tau.restype = C.c_int
        L.orc_interval_vjp_tau.argtypes = [h, _dp, _dp, _dp, _dp, _dp, _dp]
        L.orc_interval_vjp_tau.restype = None
        i64 = C.c_int64
        L.orc_collide_range.argtypes = [h, _dp, _dp, _dp, i64, i64]
        L.orc_collide_range.restype = None
        L.orc_stream_range.argtypes = [h, _dp, _dp, _dp, i64, i64]
        L.orc_stream_range.restype = None
        L.orc_ports_range.argtypes = [h, _dp, i64, i64]
        L.orc_ports_range.restype = C.c_double
        L.orc_ports_vjp_range.argtypes = [h, _dp, _dp, i64, i64]
        L.orc_ports_vjp_range.restype = None
        L.orc_stream_vjp_range.argtypes = [h, _dp, _dp, i64, i64]
        L.orc_stream_vjp_range.restype = None
        L.orc_collide_vjp_range.argtypes = [h, _dp, _dp, _dp, _dp, _dp, _dp, i64, i64]
        L.orc_collide_vjp_range.restype = None
        L.orc_set_time.argtypes = [h, C.c_int64]
        L.orc_set_time.restype = None
        L.orc_wall_loads.argtypes = [h, _dp, _dp, C.c_double, _dp]
        L.orc_wall_loads.restype = C.c_int64
        L.orc_port_apply.argtypes = [h, C.c_int, _dp, _dp]
        L.orc_port_apply.restype = None
        _lib = L
    return _lib


def _p(a):
    return None if a is None else a.ctypes.data_as(_dp)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


def threads() -> int:
    return int(lib().orc_threads())


def mrt_basis(q: int):
    rows = np.empty(q * q)
    norms = np.empty(q)
    groups = np.empty(q, dtype=np.int32)
    if lib().orc_mrt_basis(q, _p(rows), _p(norms), groups.ctypes.data_as(C.POINTER(C.c_int32))) != 0:
        raise RuntimeError("basis incomplete")
    return rows.reshape(q, q), norms, groups


class Oracle:
    """FP64 restatement of one normalised problem (see lbm_oracle.h)."""

    def __init__(self, normalized_problem):
        self.problem = normalized_problem
        self._cp = normalized_problem.to_c()
        h = C.c_void_p()
        if lib().orc_create(C.addressof(self._cp), C.byref(h)) != 0:
            raise RuntimeError(lib().orc_error().decode())
        self.h = h
        cells, q, tau, fl = C.c_int64(), C.c_int32(), C.c_double(), C.c_int64()
        a = (C.c_double * 3)()
        lib().orc_info(self.h, C.byref(cells), C.byref(q), C.byref(tau), a, C.byref(fl))
        self.cells, self.q, self.tau = cells.value, q.value, tau.value
        self.fluid_cells = fl.value
        self.acceleration_lattice = tuple(a)

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_destroy(self.h)
            self.h = None

    def design(self, raw):
        raw = np.ascontiguousarray(raw, dtype=np.float64).reshape(-1)
        phi, alpha = np.empty(self.cells), np.empty(self.cells)
        lib().orc_design(self.h, _p(raw), _p(phi), _p(alpha))
        return phi, alpha

    def design_vjp(self, raw, phi_bar):
        raw = np.ascontiguousarray(raw, dtype=np.float64).reshape(-1)
        pb = np.ascontiguousarray(phi_bar, dtype=np.float64).reshape(-1)
        out = np.empty(self.cells)
        lib().orc_design_vjp(self.h, _p(raw), _p(pb), _p(out))
        return out

    def resistance_derivative(self, phi):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        out = np.empty(self.cells)
        lib().orc_resistance_derivative(self.h, _p(phi), _p(out))
        return out

    def initial(self):
        f = np.empty(self.cells * self.q)
        lib().orc_initial(self.h, _p(f))
        return f.reshape(self.cells, self.q)

    def interval(self, before, alpha):
        b = np.ascontiguousarray(before, dtype=np.float64).reshape(-1)
        al = np.ascontiguousarray(alpha, dtype=np.float64)
        out = np.empty_like(b)
        ex = lib().orc_interval(self.h, _p(b), _p(al), _p(out))
        return out.reshape(self.cells, self.q), ex

    def history(self, alpha, steps):
        al = np.ascontiguousarray(alpha, dtype=np.float64)
        f = np.empty(self.cells * self.q)
        d = Diag()
        lib().orc_history(self.h, _p(al), int(steps), _p(f), C.byref(d))
        return f.reshape(self.cells, self.q), d

    def history_trace(self, alpha, steps):
        al = np.ascontiguousarray(alpha, dtype=np.float64)
        f = np.empty(self.cells * self.q)
        mass, exch = np.empty(steps + 1), np.empty(steps + 1)
        d = Diag()
        lib().orc_history_trace(self.h, _p(al), int(steps), _p(f), C.byref(d), _p(mass), _p(exch))
        return f.reshape(self.cells, self.q), d, mass, exch

    def vector(self, phi, alpha, f):
        out = np.empty(8)
        lib().orc_vector(self.h, _p(np.ascontiguousarray(phi, dtype=np.float64)),
                         _p(np.ascontiguousarray(alpha, dtype=np.float64)),
                         _p(np.ascontiguousarray(f, dtype=np.float64)), _p(out))
        return out

    def vector_vjp(self, phi, alpha, f, w):
        fb = np.empty(self.cells * self.q)
        ab, pb = np.empty(self.cells), np.empty(self.cells)
        w8 = np.zeros(8)
        w8[: len(w)] = w
        lib().orc_vector_vjp(self.h, _p(np.ascontiguousarray(phi, dtype=np.float64)),
                             _p(np.ascontiguousarray(alpha, dtype=np.float64)),
                             _p(np.ascontiguousarray(f, dtype=np.float64)), _p(w8), _p(fb), _p(ab), _p(pb))
        return fb.reshape(self.cells, self.q), ab, pb

    def interval_vjp(self, before, alpha, after_bar):
        b = np.ascontiguousarray(before, dtype=np.float64).reshape(-1)
        ab_ = np.ascontiguousarray(after_bar, dtype=np.float64).reshape(-1)
        fb = np.empty_like(b)
        abar = np.empty(self.cells)
        lib().orc_interval_vjp(self.h, _p(b), _p(np.ascontiguousarray(alpha, dtype=np.float64)), _p(ab_), _p(fb),
                               _p(abar))
        return fb.reshape(self.cells, self.q), abar

    def gradient(self, raw, weights, steps=None, mode="horizon", K=0, tol=1e-12, max_iter=200000):
        raw = np.ascontiguousarray(raw, dtype=np.float64).reshape(-1)
        w8 = np.zeros(8)
        w8[: len(weights)] = weights
        grad = np.empty(self.cells)
        resp = np.empty(8)
        rep = GradReport()
        steps = self.problem.step_count if steps is None else steps
        m = {"horizon": 0, "steady": 1, "time_average": 2}[mode]
        st = lib().orc_gradient(self.h, _p(raw), _p(w8), int(steps), m, int(K),
                                float(tol), int(max_iter), _p(grad), _p(resp), C.byref(rep))
        return grad, resp, rep, st

    def wall_loads(self, before, alpha, pressure_datum_pa=0.0):
        """Wall momentum-exchange forces [n,3] (N) of the interval starting at `before`."""
        b = np.ascontiguousarray(before, dtype=np.float64).reshape(-1)
        al = np.ascontiguousarray(alpha, dtype=np.float64)
        n = lib().orc_wall_loads(self.h, _p(b), _p(al), float(pressure_datum_pa), None)
        out = np.empty((n, 3))
        lib().orc_wall_loads(self.h, _p(b), _p(al), float(pressure_datum_pa), _p(out))
        return out

    def set_tau(self, tau):
        """Per-cell relaxation times of the BGK collision (None: uniform)."""
        self._tau = None if tau is None else np.ascontiguousarray(tau, dtype=np.float64).reshape(-1)
        if lib().orc_set_tau(self.h, _p(self._tau)) != 0:
            raise RuntimeError("per-cell tau needs the BGK collision")

    def interval_vjp_tau(self, before, alpha, after_bar):
        b = np.ascontiguousarray(before, dtype=np.float64).reshape(-1)
        ab_ = np.ascontiguousarray(after_bar, dtype=np.float64).reshape(-1)
        fb = np.empty_like(b)
        abar, tbar = np.empty(self.cells), np.empty(self.cells)
        lib().orc_interval_vjp_tau(self.h, _p(b), _p(np.ascontiguousarray(alpha, dtype=np.float64)), _p(ab_),
                                   _p(fb), _p(abar), _p(tbar))
        return fb.reshape(self.cells, self.q), abar, tbar

    def set_time(self, t_index: int):
        """Port values of the reconstruction producing state t_index."""
        lib().orc_set_time(self.h, int(t_index))

    def port_apply(self, k, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        out = np.empty_like(f)
        lib().orc_port_apply(self.h, int(k), _p(f), _p(out))
        return out
