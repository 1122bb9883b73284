"""A slab backend over the FP64 oracle (test infrastructure): one rank's share
of each step computed with the oracle's cell-range pieces of interval and
interval_vjp (oracle/lbm_oracle.h).  Every array holds NaN outside the
rank's own cells and the halo slots the exchange delivers, so a slot that the
decomposition fails to provide turns the result into NaN."""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from oracle import oracle as orc

_dp = C.POINTER(C.c_double)


def _p(a):
    return a.ctypes.data_as(_dp)


class OracleSlab:
    def __init__(self, norm, slab, raw):
        self.o = orc.Oracle(norm)
        self.slab = slab
        self.q = self.o.q
        self.shape = tuple(norm.shape)
        nx, ny, nz = self.shape
        self.sx = ny * nz
        self.cells_global = self.o.cells
        self.c0, self.c1 = slab.x_begin * self.sx, slab.x_end * self.sx
        self.raw = np.ascontiguousarray(raw, dtype=np.float64).reshape(-1)
        self.phi, self.alpha = self.o.design(self.raw)
        self.dres = self.o.resistance_derivative(self.phi)
        self.solid = np.asarray(norm.solid_mask, bool).reshape(-1)
        self.own = np.zeros(self.cells_global, bool)
        self.own[self.c0:self.c1] = True
        self.lib = orc.lib()
        self.diags = []
        # lattice weights: a fluid cell at rest with zero force holds w
        self.w = np.asarray(self._weights(), dtype=np.float64)

    def _weights(self):
        if self.q == 19:
            c = np.array([[0, 0, 0], [-1, -1, 0], [-1, 0, -1], [-1, 0, 0], [-1, 0, 1], [-1, 1, 0], [0, -1, -1],
                          [0, -1, 0], [0, -1, 1], [0, 0, -1], [0, 0, 1], [0, 1, -1], [0, 1, 0], [0, 1, 1], [1, -1, 0],
                          [1, 0, -1], [1, 0, 0], [1, 0, 1], [1, 1, 0]])
            c2 = (c ** 2).sum(1)
            return np.where(c2 == 0, 1 / 3, np.where(c2 == 1, 1 / 18, 1 / 36))
        c = np.array([[0, 0, 0]] + [[a, b, d] for a in (-1, 0, 1) for b in (-1, 0, 1) for d in (-1, 0, 1)
                                    if (a, b, d) != (0, 0, 0)])
        c2 = (c ** 2).sum(1)
        return np.select([c2 == 0, c2 == 1, c2 == 2], [8 / 27, 2 / 27, 1 / 54], 1 / 216)

    def _nan(self):
        return np.full((self.cells_global, self.q), np.nan)

    def _plane_cells(self, x):
        x %= self.slab.nx
        return np.arange(x * self.sx, (x + 1) * self.sx)

    def _boundary(self, side):
        return self._plane_cells(self.slab.x_end - 1 if side == "right" else self.slab.x_begin)

    def _ghost(self, side):
        return self._plane_cells(self.slab.x_begin - 1 if side == "left" else self.slab.x_end)

    # ---------------------------------------------------------------- halos
    def halo_pack(self, kind, msg):
        src = self.post if kind == "state" else self.refl
        vals = src[np.ix_(self._boundary(msg.side), list(msg.directions))]
        return torch.from_numpy(np.ascontiguousarray(vals))

    def halo_unpack(self, kind, msg, values):
        dst = self.post if kind == "state" else self.refl
        dst[np.ix_(self._ghost(msg.side), list(msg.directions))] = values.numpy()

    # ---------------------------------------------------------------- forward
    def _diag(self, f, exchange):
        own_fluid = self.own & ~self.solid
        g = f[own_fluid]
        rho = g.sum(1)
        a = np.asarray(self.o.acceleration_lattice)
        from test_gpu_parity import macroscopic

        _, u = macroscopic(g, self.q, self.alpha[own_fluid], a)
        return [float(rho.sum()), float(exchange), float(g.min()) if g.size else np.inf,
                float((u ** 2).sum(1).max()) if g.size else 0.0, float(not np.all(np.isfinite(f[self.own])))]

    def forward_begin(self):
        f = self.o.initial()
        self.before = self._nan()
        self.before[self.own] = f[self.own]
        self.diags = [self._diag(self.before, 0.0)]

    def forward_stage(self, t):
        self.o.set_time(t + 1)
        self.post = self._nan()
        self.lib.orc_collide_range(self.o.h, _p(self.before), _p(self.alpha), _p(self.post), self.c0, self.c1)

    def forward_finish(self, t):
        after = self._nan()
        self.lib.orc_stream_range(self.o.h, _p(self.post), _p(self.before), _p(after), self.c0, self.c1)
        exch = self.lib.orc_ports_range(self.o.h, _p(after), self.c0, self.c1)
        self.before = after
        self.diags.append(self._diag(after, exch))

    def diagnostics(self):
        return np.asarray(self.diags)

    def final_state(self):
        return self.before[self.own]

    def _filled(self):
        f = np.tile(self.w, (self.cells_global, 1))
        f[self.own] = self.before[self.own]
        return f

    def responses(self):
        # other ranks' cells hold the rest state with an unbounded resistance:
        # their Brinkman velocity, force and every response term vanish
        phi = np.where(self.own, self.phi, 0.0)
        alpha = np.where(self.own, self.alpha, 1e30)
        return self.o.vector(phi, alpha, self._filled())

    # ---------------------------------------------------------------- adjoint
    def adjoint_begin(self, weights):
        fb, ab, pb = self.o.vector_vjp(self.phi, self.alpha, self._filled(), weights)
        self.lam = self._nan()
        self.lam[self.own] = fb[self.own]
        self.abar_final = np.where(self.own, ab, 0.0)
        self.phibar = np.where(self.own, pb, 0.0)
        self.abar = np.zeros(self.cells_global)
        return float(np.sum(self.lam[self.own] ** 2))

    def adjoint_stage(self):
        self.refl = self._nan()
        self.lib.orc_ports_vjp_range(self.o.h, _p(self.lam), _p(self.refl), self.c0, self.c1)

    def adjoint_finish(self, want_norm=True):
        post_bar = self._nan()
        self.lib.orc_stream_vjp_range(self.o.h, _p(self.refl), _p(post_bar), self.c0, self.c1)
        fb = self._nan()
        ab = np.zeros(self.cells_global)
        self.lib.orc_collide_vjp_range(self.o.h, _p(self.before), _p(self.alpha), _p(post_bar), _p(self.refl), _p(fb),
                                       _p(ab), self.c0, self.c1)
        self.abar[self.own] += ab[self.own]
        self.lam = fb
        return float(np.sum(self.lam[self.own] ** 2))

    def gradient(self):
        phibar = self.phibar + (self.abar + self.abar_final) * self.dres
        phibar = np.where(self.own, phibar, 0.0)
        return self.o.design_vjp(self.raw, phibar)
