"""The density topology-optimisation loop: GPU forward + steady adjoint +
sensitivity per design iteration, then the CPU MMA update.

Mirrors the reference's MMA driver (crates/implexity-jobs/src/optimize/
mma_driver.rs): the objective and constraints are scaled once, at the first
iterate (``calibrate``, :199-251: s0 = 1/max(|f0|, 1e-8), s_j = 1/max(|f_j|,
1), c_j = max(1000, 10 max|s0 df0| / max|s_j df_j|)), and every step hands
the scaled values to ``MmaOptimizer::step`` (:288-345), or, with ``gcmma``,
to ``MmaOptimizer::step_gcmma`` (mma.rs:666-769), whose conservative inner
loop evaluates the true objective and constraint at each trial design (one
forward solve and the responses; no adjoint).  The design variables are the
editable cells' raw densities in [0, 1]; the constraint is the reference's
volume-fraction residual v_mean / t - 1 <= 0 with v_mean the mean design
density phi over the cells and t the target fraction (spec.rs:782-790,
problem.rs:552-573), whose gradient 1 / (N t) per cell is pulled back through
the design-map transpose (no adjoint solve).

Command line (one GPU)::

    python -m implexity_b200.optimize --shape 512 256 256 --iterations 30 --forward-steps 3000
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import workloads
from .mma import MmaOptimizer
from .problem import ContractError, normalize
from .solver import LbmSolver


class DesignLoop:
    def __init__(self, problem: dict, weights, volume_fraction: float = 0.4, mma_options: dict | None = None,
                 gcmma: bool | dict = False, adjoint_max_iterations: int = 1_000_000):
        self.norm = normalize(problem)
        self.shape = tuple(self.norm.shape)
        self.w = np.asarray(weights, float)
        self.vf = float(volume_fraction)
        self.solver = LbmSolver(self.norm)
        editable = np.asarray(self.norm.design_region, bool) & ~np.asarray(self.norm.solid_mask, bool)
        self.free = editable.reshape(self.shape)
        self.n = int(self.free.sum())
        self.cells = int(np.prod(self.shape))
        self.dv = self.norm.spacing_m ** 3
        self.opt = None  # built at the first iterate, once c is calibrated
        self.s0 = None
        self.s = None
        self.c = None
        self.mma_options = dict(mma_options or {})
        self.gcmma = gcmma
        # the Neumann count of the long C5 channel grows as the design opens
        # (89 000 at the first iterate, ~98 000 by the eighth at 512x256x256)
        self.adjoint_max_iterations = int(adjoint_max_iterations)
        self.trial_evaluations = 0

    def close(self):
        self.solver.close()
        if self.opt is not None:
            self.opt.close()

    def evaluate(self, raw: np.ndarray):
        """Objective, its gradient, the volume constraint and its gradient."""
        s = self.solver
        t0 = time.perf_counter()
        s.set_design(raw)
        d = s.forward()
        r = s.responses()
        t1 = time.perf_counter()
        g, rep = s.gradient(self.w, mode="steady", tolerance=1e-8, lambda_storage=self.norm.options.storage,
                            check_every=100, max_iterations=self.adjoint_max_iterations)
        t2 = time.perf_counter()
        v_mean = r[5] / (self.cells * self.dv)
        dres = s.design_vjp(np.full(self.shape, 1.0 / (self.cells * self.vf)))
        t3 = time.perf_counter()
        f0 = float(np.dot(self.w, r))
        timing = {"forward_s": t1 - t0, "adjoint_s": t2 - t1, "volume_s": t3 - t2, "forward_ms_device": d.device_ms,
                  "adjoint_ms_device": rep.adjoint_ms, "adjoint_iterations": rep.iterations}
        return f0, g.reshape(self.shape), v_mean / self.vf - 1.0, dres.reshape(self.shape), timing

    def calibrate(self, f0: float, df0: np.ndarray, fs: np.ndarray, dfs: np.ndarray):
        """Scaling of mma_driver.rs:199-251, at the first iterate."""
        self.s0 = 1.0 / max(abs(f0), 1e-8)
        self.s = 1.0 / np.maximum(np.abs(fs), 1.0)
        g0 = float(np.max(np.abs(self.s0 * df0))) if df0.size else 0.0
        c = []
        for j in range(len(fs)):
            gj = float(np.max(np.abs(self.s[j] * dfs[j]))) if dfs[j].size else 0.0
            c.append(max(1000.0, 10.0 * g0 / gj) if gj > 0.0 else 1000.0)
        self.c = np.array(c)
        self.opt = MmaOptimizer(self.n, len(fs), x_min=0.0, x_max=1.0, c=self.c,
                                gcmma=self.gcmma if self.gcmma else None, **self.mma_options)

    def true_values(self, raw: np.ndarray):
        """The objective and the volume constraint of a trial design (the
        GCMMA inner loop's eval_true): forward solve and responses only.  A
        design whose evaluation is refused (admission) reads as non-finite,
        which makes GCMMA raise rho and retry."""
        s = self.solver
        self.trial_evaluations += 1
        s.set_design(raw)
        try:
            s.forward()
        except ContractError:
            return float("nan"), np.array([float("nan")])
        r = s.responses()
        con = r[5] / (self.cells * self.dv) / self.vf - 1.0
        return float(np.dot(self.w, r)), np.array([con])

    def run(self, raw0: np.ndarray, iterations: int, log=None) -> dict:
        raw = np.array(raw0, dtype=float).reshape(self.shape)
        x = raw[self.free].copy()
        xm1 = xm2 = x.copy()
        history = []
        stopped = None
        for it in range(iterations):
            t0 = time.perf_counter()
            try:
                f0, g, con, dcon, timing = self.evaluate(raw)
            except ContractError as e:
                # the reference driver fails the job when an evaluation is
                # refused (admission); the loop stops here and keeps its history
                stopped = {"iteration": it, "stopped": str(e)}
                if log:
                    log(stopped)
                break
            df0 = g[self.free]
            fs = np.array([con])
            dfs = dcon[self.free][None, :]
            if self.s0 is None:
                self.calibrate(f0, df0, fs, dfs)
            t1 = time.perf_counter()
            if self.gcmma:
                def eval_true(xt):
                    trial = raw.copy()
                    trial[self.free] = xt
                    tf0, tfs = self.true_values(trial)
                    return self.s0 * tf0, self.s * tfs

                xn = self.opt.step_gcmma(x, xm1, xm2, self.s0 * f0, self.s0 * df0, self.s * fs,
                                         (self.s[:, None] * dfs).ravel(), eval_true)
            else:
                xn = self.opt.step(x, xm1, xm2, self.s0 * f0, self.s0 * df0, self.s * fs,
                                   (self.s[:, None] * dfs).ravel())
            t2 = time.perf_counter()
            info = self.opt.last
            rec = {"iteration": it, "objective": f0, "volume_fraction": (con + 1.0) * self.vf,
                   "kkt_residual": info.kkt_residual, "max_move": float(np.max(np.abs(xn - x))),
                   "mma_s": t2 - t1, "mma_newton_steps": info.newton_steps, "wall_s": t2 - t0,
                   "gcmma_inner": info.inner_iterations, "conservative": info.conservative, **timing}
            history.append(rec)
            if log:
                log(rec)
            xm2, xm1, x = xm1, x, xn
            raw[self.free] = x
        return {"history": history, "final_design": raw, "stopped": stopped}


def c5_problem(shape=(512, 256, 256), forward_steps=3000, storage="float32"):
    """The full-loop workload: D3Q19 TRT channel, conic filter of radius 2 cells."""
    return workloads.channel_problem(shape=shape, steps=forward_steps, collision="trt", storage=storage,
                                     box_half_width=0, filter_radius_cells=2.0)


def c5_initial_design(shape, seed=0):
    """rho0 = 0.5 + 0.05 U(0, 1) noise (seeded)."""
    return 0.5 + 0.05 * np.random.default_rng(seed).uniform(0.0, 1.0, size=shape)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--shape", type=int, nargs=3, default=[512, 256, 256])
    ap.add_argument("--iterations", type=int, default=30)
    ap.add_argument("--forward-steps", type=int, default=3000)
    ap.add_argument("--storage", choices=["float32", "float16"], default="float32")
    ap.add_argument("--volume-fraction", type=float, default=0.4)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--gcmma", action="store_true", help="conservative GCMMA steps (MmaOptimizer::step_gcmma)")
    a = ap.parse_args()
    shape = tuple(a.shape)
    loop = DesignLoop(c5_problem(shape, a.forward_steps, a.storage), workloads.objective_weights(), a.volume_fraction,
                      gcmma=a.gcmma)
    try:
        out = loop.run(c5_initial_design(shape, a.seed), a.iterations,
                       log=lambda r: print(json.dumps(r), flush=True))
    finally:
        loop.close()
    h = out["history"]
    print(json.dumps({"design_loop": list(shape), "storage": a.storage, "iterations": len(h),
                      "stopped": out["stopped"],
                      "objective": [r["objective"] for r in h], "volume_fraction": [r["volume_fraction"] for r in h],
                      "wall_s_per_iteration": [r["wall_s"] for r in h], "mma_s": [r["mma_s"] for r in h]}))


if __name__ == "__main__":
    main()
