"""Generates the golden fixtures of tests/golden/ from an independent numpy
restatement of the reference's LBM density-design path.

This restatement is written separately from the C++ oracle (oracle/), vector
by vector from the reference's formulas, so that the two pin each other:

* d3q19.rs:29-59           velocity set, weights, opposites
* solver.rs:84-136         pull streaming with halfway bounce-back
* solver.rs:190-210,298-322 Guo-Brinkman BGK collision (implicit half-step u)
* moving/collision.rs:457-488 TRT pair collision (magic 3/16)
* ports.rs:343-406          legacy-moment port reconstruction
* design.rs:109-216,282-294 conic filter, tanh projection, RAMP resistance
* solver.rs:835-893         responses (+ pressure drop, viscous dissipation)
* solver.rs:593-601         initial populations

The gradients in the fixtures are complex-step derivatives of this
restatement (no adjoint: d J / d raw_x = Im J(raw + i h e_x) / h with
h = 1e-30, exact to rounding), so they check the oracle's discrete adjoint
against an independent forward model.

Cases:
  template_bgk  the reference's own problem template (provider.rs:74-90):
                4x6x4, 10 steps, BGK, periodic x/z, body force, conic filter
                1.5 mm with projection beta 2
  channel_trt   8x6x6 channel, 12 steps, TRT, velocity inlet + pressure
                outlet, box filter
Run: python tests/golden/make_golden.py   (writes tests/golden/*.npz)
"""
from __future__ import annotations

import json
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent

C = np.array(
    [[0, 0, 0], [-1, -1, 0], [-1, 0, -1], [-1, 0, 0], [-1, 0, 1], [-1, 1, 0], [0, -1, -1], [0, -1, 0], [0, -1, 1],
     [0, 0, -1], [0, 0, 1], [0, 1, -1], [0, 1, 0], [0, 1, 1], [1, -1, 0], [1, 0, -1], [1, 0, 0], [1, 0, 1], [1, 1, 0]])
W = np.where((C != 0).sum(1) == 0, 1 / 3, np.where((C != 0).sum(1) == 1, 1 / 18, 1 / 36))
OPP = np.array([int(np.where((C == -C[q]).all(1))[0][0]) for q in range(19)])


class Model:
    def __init__(self, p: dict):
        self.shape = tuple(p["shape"])
        self.n = int(np.prod(self.shape))
        self.per = np.array(p["periodic_axes"], bool)
        self.dx, self.dt = p["spacing_m"], p["step_s"]
        self.rho_ref = p["density_kg_m3"]
        self.tau = 0.5 + 3 * p["kinematic_viscosity_m2_s"] * self.dt / self.dx**2
        self.a = np.array(p["acceleration_m_s2"], float) * self.dt**2 / self.dx
        self.solid = np.asarray(p["solid_mask"], bool).ravel()
        self.design = np.asarray(p["design_region"], bool).ravel()
        self.fixed = np.asarray(p["fixed_design"], float).ravel()
        self.dmax, self.q = p["drag_max_per_s"], p["drag_shape"]
        self.steps = p["step_count"]
        self.coll = p.get("collision", "bgk")
        self.coords = np.stack(np.unravel_index(np.arange(self.n), self.shape), 1)
        self._streaming()
        self._filter(p["topology_map"], p.get("box_half_width", 0))
        self.ports = [self._port(pt) for pt in p.get("ports", [])]

    def index(self, ijk):
        return np.ravel_multi_index(tuple(ijk.T), self.shape)

    def _streaming(self):
        # pull source of (x, q): x - c_q, or (x, opp q) when the link is blocked
        src = np.empty((self.n, 19), dtype=np.int64)
        shp = np.array(self.shape)
        for q in range(19):
            back = self.coords - C[q]
            outside = ((back < 0) | (back >= shp)) & ~self.per
            wrapped = self.index(back % shp)
            blocked = outside.any(1) | self.solid[wrapped]
            src[:, q] = np.where(blocked, np.arange(self.n) * 19 + OPP[q], wrapped * 19 + q)
        self.src = src

    def _filter(self, tm, box_hw):
        self.editable = self.design & ~self.solid
        self.beta, self.eta = tm["projection_beta"], tm["projection_eta"]
        r = tm["filter_radius_m"] / self.dx
        offs = []
        if box_hw > 0:
            rng = range(-box_hw, box_hw + 1)
            offs = [((i, j, k), 1.0) for i in rng for j in rng for k in rng]
        elif r > 0:
            reach = int(np.ceil(r))
            rng = range(-reach, reach + 1)
            for i in rng:
                for j in rng:
                    for k in rng:
                        wgt = max(r - np.sqrt(i * i + j * j + k * k), 0.0)
                        if wgt != 0:
                            offs.append(((i, j, k), wgt))
        self.rows = None
        if offs:
            shp = np.array(self.shape)
            self.rows = []
            for x in range(self.n):
                terms = []
                for off, wgt in offs:
                    s = self.coords[x] - np.array(off)
                    if (((s < 0) | (s >= shp)) & ~self.per).any():
                        continue
                    si = int(self.index((s % shp)[None])[0])
                    if self.editable[si]:
                        terms.append((si, wgt))
                self.rows.append(terms)

    def fraction(self, raw):
        raw = raw.ravel()
        phi = np.where(self.solid, 0.0, self.fixed).astype(raw.dtype)
        for x in np.where(self.editable)[0]:
            if self.rows is None:
                f = raw[x]
            else:
                den = sum(w for _, w in self.rows[x]) or 1.0
                f = sum(w * raw[s] for s, w in self.rows[x]) / den
            if self.beta > 0:
                a = np.tanh(self.beta * self.eta)
                f = (a + np.tanh(self.beta * (f - self.eta))) / (a + np.tanh(self.beta * (1 - self.eta)))
            phi[x] = f
        return phi

    def resistance(self, phi):
        return self.dt * self.dmax * self.q * (1 - phi) / (self.q + phi)

    def _port(self, pt):
        axis = "xyz".index(pt["face"][0])
        sign = 1 if pt["face"].endswith("min") else -1
        u = np.array(pt["velocity_m_s"]) * self.dt / self.dx
        rho = None
        if pt["kind"] == "pressure":
            unit = self.dx / self.dt
            rho = 1 + pt["gauge_pressure_Pa"] * 3 / (self.rho_ref * unit * unit)
        cells = np.where(np.asarray(pt["mask"], bool).ravel())[0]
        return dict(axis=axis, sign=sign, u=u, rho=rho, cells=cells)

    def reconstruct(self, f, pt):
        ax, sg = pt["axis"], pt["sign"]
        unk = np.where(C[:, ax] == sg)[0]
        out_ = np.where(C[:, ax] == -sg)[0]
        zero = np.where(C[:, ax] == 0)[0]
        t0, t1 = [d for d in range(3) if d != ax]
        v = pt["u"] - 0.5 * self.a
        compat = f[zero].sum() + 2 * f[out_].sum()
        if pt["rho"] is None:
            rho = compat / (1 - sg * v[ax])
        else:
            rho = pt["rho"]
            v = v.astype(np.result_type(v, compat))
            v[ax] = (1 - compat / rho) * sg
        prop = f[OPP[unk]] + rho * 6 * W[unk] * (C[unk] @ v)
        known = f.copy()
        known[unk] = 0
        target = np.array([rho - known.sum(), rho * v[t0] - known @ C[:, t0], rho * v[t1] - known @ C[:, t1]])
        R = np.stack([np.ones(len(unk)), C[unk, t0], C[unk, t1]]).astype(float)
        corr = R.T @ np.linalg.solve(R @ R.T, target - R @ prop)
        out = f.copy()
        out[unk] = prop + corr
        return out

    def macroscopic(self, f, alpha):
        rho = f.sum(1)
        u = (f @ C / rho[:, None] + 0.5 * self.a) / (1 + 0.5 * alpha[:, None])
        F = rho[:, None] * (self.a - alpha[:, None] * u)
        return rho, u, F

    def collide(self, f, alpha):
        rho, u, F = self.macroscopic(f, alpha)
        cu, cf = u @ C.T, F @ C.T
        usq, uf = (u * u).sum(1)[:, None], (u * F).sum(1)[:, None]
        eq = rho[:, None] * W * (1 + 3 * cu + 4.5 * cu * cu - 1.5 * usq)
        src = W * (3 * cf - 3 * uf + 9 * cu * cf)
        om = 1 / self.tau
        if self.coll == "bgk":
            return f - om * (f - eq) + (1 - om / 2) * src
        tp = self.tau - 0.5
        omm = 1 / (0.5 + (3 / 16) / tp)
        fp, fm = 0.5 * (f + f[:, OPP]), 0.5 * (f - f[:, OPP])
        ep, em = 0.5 * (eq + eq[:, OPP]), 0.5 * (eq - eq[:, OPP])
        sp, sm = 0.5 * (src + src[:, OPP]), 0.5 * (src - src[:, OPP])
        return f - om * (fp - ep) - omm * (fm - em) + (1 - om / 2) * sp + (1 - omm / 2) * sm

    def initial(self):
        f = np.tile(W - 1.5 * W * (C @ self.a), (self.n, 1))
        f[self.solid] = W
        return f

    def step(self, f, alpha):
        post = self.collide(f, alpha)
        flat = post.ravel()
        after = flat[self.src].copy()
        after[self.solid] = f[self.solid]
        exch = 0.0
        for pt in self.ports:
            for x in pt["cells"]:
                new = self.reconstruct(after[x], pt)
                exch += (new - after[x]).sum()
                after[x] = new
        return after, exch

    def run(self, alpha, steps=None):
        f = self.initial()
        mass = [f[~self.solid].sum()]
        exch = []
        for _ in range(self.steps if steps is None else steps):
            f, e = self.step(f, alpha)
            exch.append(e)
            mass.append(f[~self.solid].sum())
        return f, np.array(mass), np.array(exch)

    def responses(self, phi, alpha, f):
        fl = ~self.solid
        rho, u, F = self.macroscopic(f, alpha)
        vel = self.dx / self.dt
        U = np.where(fl[:, None], u, 0) * vel
        R = rho * self.rho_ref
        usq = (U * U).sum(1)
        dv = self.dx**3
        nf = fl.sum()
        out = np.zeros(8, dtype=np.result_type(f, alpha))
        out[:3] = U.sum(0) / nf
        out[3] = 0.5 * (R * usq * fl).sum() * dv
        out[4] = (R * alpha / self.dt * usq * fl).sum() * dv
        out[5] = phi.sum() * dv
        inl = [x for pt in self.ports if pt["rho"] is None for x in pt["cells"]]
        outl = [x for pt in self.ports if pt["rho"] is not None for x in pt["cells"]]
        if inl and outl:
            p = self.rho_ref * (rho - 1) * vel * vel / 3
            out[6] = p[inl].mean() - p[outl].mean()
        k = 1 - 0.5 / self.tau
        nu = (self.tau - 0.5) / 3
        M2 = np.einsum("xq,qa,qb->xab", f, C, C)
        Pi = M2 - rho[:, None, None] * (np.eye(3) / 3 + np.einsum("xa,xb->xab", u, u))
        T = 0.5 * (np.einsum("xa,xb->xab", u, F) + np.einsum("xa,xb->xab", F, u))
        sig = -k * (Pi + T)
        phi_v = (sig * sig).sum((1, 2)) / (2 * rho * nu)
        out[7] = (phi_v * fl).sum() * self.rho_ref * self.dx**5 / self.dt**3
        return out

    def objective(self, raw, w):
        phi = self.fraction(raw)
        alpha = self.resistance(phi)
        f, _, _ = self.run(alpha)
        return w @ self.responses(phi, alpha, f)


def template_problem():
    shape = (4, 6, 4)
    n = int(np.prod(shape))
    return {
        "shape": list(shape), "spacing_m": 0.001, "step_s": 0.1, "step_count": 10,
        "density_kg_m3": 1000.0, "kinematic_viscosity_m2_s": 1e-6,
        "acceleration_m_s2": [1e-5, 0.0, 0.0], "periodic_axes": [True, False, True],
        "solid_mask": np.zeros(shape, bool), "design_region": np.ones(shape, bool),
        "fixed_design": np.ones(shape), "drag_max_per_s": 10.0, "drag_shape": 0.1, "mach_limit": 0.1,
        "history_byte_budget": 16_000_000,
        "topology_map": {"filter_radius_m": 0.0015, "projection_beta": 2.0, "projection_eta": 0.5},
        "ports": [], "collision": "bgk", "n": n,
    }


def channel_problem():
    shape = (8, 6, 6)
    nx, ny, nz = shape
    dt = 0.1
    inlet = np.zeros(shape, bool)
    inlet[0, 1:-1, 1:-1] = True
    outlet = np.zeros(shape, bool)
    outlet[-1, 1:-1, 1:-1] = True
    design = np.zeros(shape, bool)
    design[1:-1] = True
    solid = np.zeros(shape, bool)
    solid[3, 2, 2] = True
    design &= ~solid
    return {
        "shape": list(shape), "spacing_m": 0.001, "step_s": dt, "step_count": 12,
        "density_kg_m3": 1000.0, "kinematic_viscosity_m2_s": 1e-6,
        "acceleration_m_s2": [0.0, 0.0, 0.0], "periodic_axes": [False, False, False],
        "solid_mask": solid, "design_region": design, "fixed_design": np.ones(shape),
        "drag_max_per_s": 1.0, "drag_shape": 0.1, "mach_limit": 0.2, "history_byte_budget": 10**9,
        "topology_map": {"filter_radius_m": 0.0, "projection_beta": 0.0, "projection_eta": 0.5},
        "box_half_width": 1,
        "ports": [
            {"id": "in", "kind": "velocity", "face": "xmin", "mask": inlet, "velocity_m_s": [0.04 * 0.001 / dt, 0, 0]},
            {"id": "out", "kind": "pressure", "face": "xmax", "mask": outlet, "velocity_m_s": [0.0, 0.0, 0.0],
             "gauge_pressure_Pa": 0.0},
        ],
        "collision": "trt",
    }


def make(name, p, seed, weights, fd_cells):
    m = Model(p)
    raw = np.random.default_rng(seed).uniform(0.05, 0.95, size=p["shape"])
    phi = m.fraction(raw)
    alpha = m.resistance(phi)
    f, mass, exch = m.run(alpha)
    resp = m.responses(phi, alpha, f)
    w = np.asarray(weights, float)
    grad = np.zeros(m.n)
    h = 1e-30
    for x in fd_cells:
        z = raw.ravel().astype(complex)
        z[x] += 1j * h
        grad[x] = m.objective(z, w).imag / h
    meta = {k: v for k, v in p.items() if not isinstance(v, np.ndarray) and k != "ports"}
    np.savez_compressed(
        HERE / f"{name}.npz", raw=raw, phi=phi, alpha=alpha, final=f, mass=mass, exchange=exch, responses=resp,
        weights=w, fd_cells=np.asarray(fd_cells), fd_grad=grad[fd_cells], meta=json.dumps(meta),
    )
    print(name, "responses", resp, "fd", grad[fd_cells][:4])


if __name__ == "__main__":
    tp = template_problem()
    make("template_bgk", tp, 11, [1e3, 0, 0, 1e9, 1e9, 0, 0, 0], list(range(0, tp["n"], 3)))
    cp = channel_problem()
    make("channel_trt", cp, 12, [0, 0, 0, 0, 0, 0, 1.0, 1e6], list(range(0, 8 * 36, 7)))
