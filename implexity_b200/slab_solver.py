"""One x-slab of a problem on one GPU: the backend of implexity_b200.slabs.SlabDriver
over the CUDA library's slab entry points (lbm_create_slab, lbm_slab_*,
lbm_halo_*; include/lbm_b200.h).

Halo messages travel as CUDA tensors between ranks (NCCL point-to-point in
TorchComm): lbm_halo_pack fills a tensor on the library's stream and returns
once it is complete; a tensor that arrived is unpacked after torch's stream
has finished receiving it.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _abi
from .problem import NormalizedProblem, normalize
from .slabs import HaloMessage, Slab
from .solver import _dp, _raise

KIND = {"state": 0, "adjoint": 1}
SIDE = {"left": 0, "right": 1}


class SlabSolver:
    """The handle of one slab (owned planes plus ghost planes)."""

    def __init__(self, problem: dict | NormalizedProblem, slab: Slab, halo: int = 1, device=None):
        import torch

        self.problem = problem if isinstance(problem, NormalizedProblem) else normalize(problem)
        self.slab = slab
        self.lib = _abi.load()
        self._cp = self.problem.to_c()
        h = C.c_void_p()
        st = self.lib.lbm_create_slab(C.byref(self._cp), slab.x_begin, slab.x_end, int(halo), C.byref(h))
        if st != _abi.LBM_OK:
            _raise(st, self.lib.lbm_last_error(None).decode())
        self.h = h
        info = _abi.Info()
        self.lib.lbm_info(self.h, C.byref(info))
        self.q = int(info.q)
        self.cells = int(info.cells)
        nx, ny, nz = self.problem.shape
        self.sx = ny * nz
        self.nx_local = self.cells // self.sx
        self.cells_global = nx * ny * nz
        # the local planes in global order (ghost planes wrap for periodic x)
        self.hl = self._left_ghosts(halo)
        self.planes = [(slab.x_begin - self.hl + p) % nx for p in range(self.nx_local)]
        self.device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
        self.bytes = {}
        for kind in KIND:
            b = C.c_size_t()
            self._check(self.lib.lbm_halo_bytes(self.h, KIND[kind], C.byref(b)))
            self.bytes[kind] = int(b.value)
        self.diags = []

    def _left_ghosts(self, halo):
        s = self.slab
        return halo if s.periodic_x else min(halo, s.x_begin)

    def _check(self, st):
        if st != _abi.LBM_OK:
            _raise(st, self.lib.lbm_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.lbm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def local(self, field: np.ndarray) -> np.ndarray:
        """The slab's planes of a whole-problem field (x first)."""
        f = np.asarray(field).reshape(self.problem.shape[0], -1)
        return np.ascontiguousarray(f[self.planes]).reshape(self.nx_local, *self.problem.shape[1:])

    # -- design
    def set_design(self, raw_global: np.ndarray):
        r = self.local(np.asarray(raw_global, dtype=np.float64))
        self._check(self.lib.lbm_set_design(self.h, _dp(r), r.size))

    # -- halos
    def halo_pack(self, kind, msg: HaloMessage):
        import torch

        buf = torch.empty(self.bytes[kind], dtype=torch.uint8, device=self.device)
        self._check(self.lib.lbm_halo_pack(self.h, KIND[kind], SIDE[msg.side], C.c_void_p(buf.data_ptr())))
        return buf

    def halo_unpack(self, kind, msg: HaloMessage, buf):
        import torch

        torch.cuda.current_stream(self.device).synchronize()
        self._check(self.lib.lbm_halo_unpack(self.h, KIND[kind], SIDE[msg.side], C.c_void_p(buf.data_ptr())))

    # -- forward
    def _diag(self, fn):
        d = _abi.SlabDiag()
        self._check(fn(self.h, C.byref(d)))
        self.diags.append([d.mass, d.exchange, d.minimum_population, d.maximum_speed2, float(d.nonfinite)])

    def forward_begin(self):
        self.diags = []
        self._check(self.lib.lbm_slab_begin(self.h))

    def forward_stage(self, t):
        pass

    def forward_finish(self, t):
        self._diag(self.lib.lbm_slab_step)

    exchange_before_end = True
    # the initial state is written into the slots each cell pulls from, the
    # ghost planes' included: the first step needs no exchange (and the
    # boundary slots a neighbour would send hold nothing yet)
    exchange_before_first_step = False

    def forward_end(self):
        self._diag(self.lib.lbm_slab_inspect)

    def diagnostics(self):
        return np.asarray(self.diags)

    def responses(self):
        out = np.empty(_abi.N_RESPONSES)
        self._check(self.lib.lbm_responses(self.h, _dp(out)))
        return out

    def populations(self):
        """The slab's local state (owned and ghost cells), f[cell, q]."""
        out = np.empty(self.cells * self.q)
        self._check(self.lib.lbm_get_populations(self.h, _dp(out), out.size))
        return out.reshape(self.cells, self.q)

    def owned_cells(self):
        return slice(self.hl * self.sx, (self.hl + self.slab.x_end - self.slab.x_begin) * self.sx)

    # -- steady adjoint
    def adjoint_begin(self, weights):
        w = np.zeros(_abi.N_RESPONSES)
        w[: len(weights)] = weights
        n2 = C.c_double()
        self._check(self.lib.lbm_slab_adjoint_begin(self.h, _dp(w), C.byref(n2)))
        return n2.value

    def adjoint_stage(self):
        pass

    def adjoint_finish(self, want_norm=True):
        n2 = C.c_double()
        self._check(self.lib.lbm_slab_adjoint_step(self.h, C.byref(n2) if want_norm else None))
        return n2.value if want_norm else 0.0

    def gradient(self):
        g = np.empty(self.cells)
        self._check(self.lib.lbm_slab_gradient(self.h, _dp(g), g.size))
        out = np.zeros((self.problem.shape[0], self.sx))
        np.add.at(out, self.planes, g.reshape(self.nx_local, self.sx))
        return out.ravel()
