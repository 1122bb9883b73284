"""The unsteady workload with a stage objective: memory and recompute of the
checkpointed adjoint for several checkpoint intervals K.

D3Q27 TRT channel with a pulsatile plug inlet u(t) = 0.04 (1 + 0.5 sin(2 pi t /
(1000 dt))) (lattice units), 4000 steps, objective = the time average of the
viscous dissipation (or the weighted responses of the channel objective)
over the states 1..T.  The adjoint is the
horizon adjoint with a checkpoint every K steps (scan.rs Every(K)); when a
segment's per-step records do not fit in device memory, each segment is split
once more (a second checkpoint level).  For every K the report gives the
device bytes of checkpoints + records, the recomputed forward steps and the
device times; the binomial schedule (revolve) with a given number of stored
states is reported the same way.

Command line (one GPU)::

    python -m implexity_b200.unsteady --shape 192 192 192 --steps 4000 --K 50 200 800 --snapshots 10 40
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import workloads
from .problem import normalize
from .solver import LbmSolver


def weights(objective: str) -> np.ndarray:
    """'dissipation': response 7 alone; 'channel': pressure drop + dissipation."""
    if objective == "dissipation":
        w = np.zeros(8)
        w[7] = 1.0
        return w
    return workloads.objective_weights()


def run(shape, steps, Ks, period_steps=1000, storage="float32", seed=0, objective="dissipation", log=print,
        snapshots=()):
    prob = workloads.pulsatile_problem(shape=tuple(shape), steps=steps, lattice="D3Q27", period_steps=period_steps,
                                       storage=storage)
    norm = normalize(prob)
    raw = workloads.uniform_design(tuple(shape), seed)
    w = weights(objective)
    out = []
    with LbmSolver(norm) as s:
        s.set_design(raw)
        t0 = time.perf_counter()
        d = s.forward()
        fwd_wall = time.perf_counter() - t0
        avg = s.time_average()
        j = float(np.dot(w, avg))
        base = {"workload": "pulsatile_d3q27", "shape": list(shape), "steps": steps, "storage": storage,
                "objective": objective,
                "objective_time_average": j, "forward_ms": d.device_ms, "forward_wall_s": fwd_wall,
                "forward_mlups": s.cells * steps / (d.device_ms / 1e3) / 1e6}
        log(json.dumps(base))
        g_first = None
        for K in Ks:
            t0 = time.perf_counter()
            g, rep = s.gradient(w, mode="horizon", checkpoint_every=K, objective="time_average", lambda_storage=storage)
            wall = time.perf_counter() - t0
            if g_first is None:
                g_first = g
            rec = {"K": K, "peak_state_GB": rep.peak_state_bytes / 1e9, "forward_recomputed": rep.forward_recomputed,
                   "adjoint_steps": rep.iterations, "recompute_ms": rep.forward_ms, "adjoint_ms": rep.adjoint_ms,
                   "sensitivity_ms": rep.sensitivity_ms, "wall_s": wall,
                   "adjoint_mlups": s.cells * rep.iterations / (rep.adjoint_ms / 1e3) / 1e6 if rep.adjoint_ms else None,
                   "grad_rel_l2_vs_first_K": float(np.linalg.norm(g - g_first) / np.linalg.norm(g_first))}
            log(json.dumps(rec))
            out.append(rec)
        for S in snapshots:
            t0 = time.perf_counter()
            g, rep = s.gradient(w, mode="horizon", checkpointing="binomial", snapshots=S, objective="time_average",
                                lambda_storage=storage)
            wall = time.perf_counter() - t0
            rec = {"binomial_snapshots": S, "peak_state_GB": rep.peak_state_bytes / 1e9,
                   "forward_recomputed": rep.forward_recomputed, "adjoint_steps": rep.iterations,
                   "recompute_ms": rep.forward_ms, "adjoint_ms": rep.adjoint_ms, "wall_s": wall,
                   "grad_rel_l2_vs_first_K": (float(np.linalg.norm(g - g_first) / np.linalg.norm(g_first))
                                              if g_first is not None else None)}
            log(json.dumps(rec))
            out.append(rec)
    return base, out


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--shape", type=int, nargs=3, default=[192, 192, 192])
    ap.add_argument("--steps", type=int, default=4000)
    ap.add_argument("--K", type=int, nargs="+", default=[50, 200, 800])
    ap.add_argument("--period-steps", type=int, default=1000)
    ap.add_argument("--storage", choices=["float32", "float16"], default="float32")
    ap.add_argument("--objective", choices=["dissipation", "channel"], default="dissipation")
    ap.add_argument("--snapshots", type=int, nargs="*", default=[],
                    help="also run the binomial schedule with these numbers of stored states")
    a = ap.parse_args()
    run(a.shape, a.steps, a.K, a.period_steps, a.storage, objective=a.objective, snapshots=a.snapshots)


if __name__ == "__main__":
    main()
