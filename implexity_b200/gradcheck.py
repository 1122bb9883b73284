"""Finite-difference checks of the design gradient along seeded directions.

Restates the checks of implexity-ad's gradcheck (crates/implexity-ad/src/
gradcheck.rs): ``central_difference`` (:218-232) taken along a direction d
instead of one coordinate, (J(x + h d) - J(x - h d)) / 2h, compared with the
adjoint directional derivative g.d; and ``taylor_test`` (:246-291), which
checks that the remainder |J(x + h d) - J(x) - h g.d| falls at second order
as h halves.  Directions are standard-normal vectors from numpy's PCG64
generator seeded seed, seed+1, ... (one per direction), restricted to the
editable cells (the gradient is zero elsewhere) whose perturbed design stays
in [0, 1] (the design contract).  The products g.d are FP64 sums on the host.

The objective J is sum_k w_k r_k over the eight responses of the final state
after the problem's step count, evaluated by the GPU forward step; g comes
from the GPU adjoint (horizon: the exact discrete gradient of J at that
state; steady: the fixed-point adjoint, which differs from J's gradient by
the distance of the forward state from steady state).

Command line (one GPU)::

    python -m implexity_b200.gradcheck --config channel128_trt --directions 8 --step 1e-4
"""
from __future__ import annotations

import argparse
import json
import math
import time
from dataclasses import asdict, dataclass

import numpy as np

from . import workloads
from .problem import normalize
from .solver import LbmSolver


@dataclass
class DirectionResult:
    seed: int
    fd: float            # central difference along d
    ad: float            # g . d from the adjoint gradient
    rel_error: float     # |fd - ad| / max(|fd|, |ad|)


@dataclass
class TaylorReport:
    """taylor_test (gradcheck.rs:246-291) along one direction."""

    steps: list
    remainders: list
    orders: list
    consecutive_second_order: int
    passed: bool


def objective(solver: LbmSolver, raw: np.ndarray, weights: np.ndarray) -> float:
    """J(raw) = w . responses after the problem's forward horizon."""
    solver.set_design(raw)
    solver.forward()
    return float(np.dot(weights, solver.responses()))


def directions(raw: np.ndarray, editable: np.ndarray, count: int, seed: int, reach: float):
    """Seeded standard-normal directions on the editable cells.  The design
    contract keeps raw in [0, 1], so a component is zeroed where raw +- reach d
    would leave that interval."""
    for k in range(count):
        d = np.random.default_rng(seed + k).standard_normal(raw.shape)
        inside = (raw - reach * np.abs(d) >= 0.0) & (raw + reach * np.abs(d) <= 1.0)
        yield seed + k, np.where(editable & inside, d, 0.0)


def directional_check(solver: LbmSolver, raw: np.ndarray, weights: np.ndarray, gradient: np.ndarray,
                      editable: np.ndarray, count: int = 8, seed: int = 0, step: float = 1e-4):
    """Central differences along `count` seeded directions against g.d."""
    out = []
    for s, d in directions(raw, editable, count, seed, step):
        jp = objective(solver, raw + step * d, weights)
        jm = objective(solver, raw - step * d, weights)
        fd = (jp - jm) / (2.0 * step)
        ad = math.fsum((gradient * d).ravel())
        den = max(abs(fd), abs(ad), 1e-300)
        out.append(DirectionResult(s, fd, ad, abs(fd - ad) / den))
    return out


def taylor_test(solver: LbmSolver, raw: np.ndarray, weights: np.ndarray, gradient: np.ndarray,
                direction: np.ndarray, h0: float, halvings: int = 4, required: int = 2) -> TaylorReport:
    """Remainder orders of J(x + h d) - J(x) - h g.d for h = h0, h0/2, ...

    A halving counts when its order lies in [1.8, 2.2] and the smaller
    remainder is above the noise floor 1e3 eps max(|J|, 1); the test passes
    with `required` consecutive such halvings ending at the last one above
    the floor (gradcheck.rs:268-288)."""
    j0 = objective(solver, raw, weights)
    slope = math.fsum((gradient * direction).ravel())
    floor = 1e3 * np.finfo(float).eps * max(abs(j0), 1.0)
    steps, rem = [], []
    h = h0
    for _ in range(halvings + 1):
        jh = objective(solver, raw + h * direction, weights)
        steps.append(h)
        rem.append(abs(jh - j0 - h * slope))
        h *= 0.5
    orders = [math.log2(rem[k] / rem[k + 1]) if rem[k + 1] > 0 and rem[k] > 0 else float("nan")
              for k in range(len(rem) - 1)]
    last = None
    for k in range(len(orders) - 1, -1, -1):
        if rem[k + 1] > floor:
            last = k
            break
    best = 0
    if last is not None:
        for k in range(last, -1, -1):
            if rem[k + 1] > floor and 1.8 <= orders[k] <= 2.2:
                best += 1
            else:
                break
    return TaylorReport(steps, rem, orders, best, best >= required)


def run(config: str, count: int, step: float, seed: int, mode: str, checkpoint_every: int,
        tolerance: float, storage: str = "float32") -> dict:
    """The gradient check of a bench workload; returns a JSON-ready report."""
    shape = workloads.CONFIGS[config][0]
    prob = workloads.config_problem(config, storage=storage)
    norm = normalize(prob)
    raw = workloads.config_design(config, 0)
    w = workloads.objective_weights()
    editable = (np.asarray(norm.design_region, bool) & ~np.asarray(norm.solid_mask, bool)).reshape(shape)
    t0 = time.perf_counter()
    with LbmSolver(norm) as s:
        s.set_design(raw)
        s.forward()
        g, rep = s.gradient(w, mode=mode, checkpoint_every=checkpoint_every, tolerance=tolerance,
                            lambda_storage=storage)
        res = directional_check(s, raw, w, g, editable, count=count, seed=seed, step=step)
    return {
        "gradcheck": config,
        "mode": mode,
        "storage": storage,
        "step": step,
        "directions": [asdict(r) for r in res],
        "max_rel_error": max(r.rel_error for r in res),
        "adjoint_iterations": rep.iterations,
        "adjoint_residual": rep.residual,
        "wall_s": time.perf_counter() - t0,
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--config", default="channel128_trt")
    ap.add_argument("--directions", type=int, default=8)
    ap.add_argument("--step", type=float, default=1e-4)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--mode", choices=["horizon", "steady"], default="horizon")
    ap.add_argument("--checkpoint-every", type=int, default=100)
    ap.add_argument("--tolerance", type=float, default=1e-8)
    ap.add_argument("--storage", choices=["float32", "float16"], default="float32")
    a = ap.parse_args()
    print(json.dumps(run(a.config, a.directions, a.step, a.seed, a.mode, a.checkpoint_every, a.tolerance,
                         a.storage)))


if __name__ == "__main__":
    main()
