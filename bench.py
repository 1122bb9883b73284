"""Benchmark: MLUPS of one design iteration (forward + steady discrete adjoint +
sensitivity) of the differentiable D3Q19 TRT lattice-Boltzmann channel.

Workload (default): 256x128x128 cells, D3Q19 TRT (tau 0.8, magic 3/16), plug
inlet u = 0.05, constant-density outlet, halfway bounce-back walls, seeded
uniform design smoothed by a 3x3x3 box filter, RAMP q = 0.1 to alpha in
[0, 0.1]; 3000 forward steps, then the steady adjoint to relative residual
1e-8 and the design-map transpose.  One bench "step" is one such design
iteration.  The 128^3 channel (5000 forward steps) and the MRT sphere
workload run with --config.

MLUPS = cells * (forward steps + adjoint iterations) / time / 1e6.
``value`` uses the device time of the stepping kernels (CUDA events on the
library's stream, design resident in HBM); ``e2e`` is the wall time of the
public API call sequence with the design uploaded from host memory and the
gradient read back every step.  The FP32 population arrays (320 MB at
256x128x128, 160 MB at 128^3) exceed the 126 MB L2, so no explicit L2 flush
is needed between steps.

``--impl reference`` times the CPU oracle (FP64 C++ restatement of the
reference's Rust path, all host threads) on a bounded sample of the same
workload.  With N GPUs (torchrun) every rank runs an independent replica:
the solver does not shard, so ``scaling`` is weak.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

from implexity_b200.workloads import CONFIGS

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

FWD_BYTES = {  # algorithmic bytes per cell update: 2 Q s_f + 4 (alpha)
    ("float32", 19): 2 * 19 * 4 + 4,
    ("float16", 19): 2 * 19 * 2 + 4,
    ("float32", 27): 2 * 27 * 4 + 4,
    ("float16", 27): 2 * 27 * 2 + 4,
}


def adj_bytes(q, s_lam):
    # record (rho-1, u) 16 B + alpha 4 B + lambda read+write 2 Q s + abar read+write 8 B
    return 16 + 4 + 2 * q * s_lam + 8


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic(kernel_tag: str):
    """Per-cell DRAM traffic of a stepping kernel from the committed ncu
    summary (profiles/<kernel_tag>.md, line 'dram_bytes_per_cell: X')."""
    p = ROOT / "profiles" / f"{kernel_tag}.md"
    if not p.exists():
        return None
    for line in p.read_text().splitlines():
        if line.strip().startswith("dram_bytes_per_cell:"):
            try:
                return float(line.split(":", 1)[1].split()[0])
            except ValueError:
                return None
    return None


class Clocks:
    """nvidia-smi sampling during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.path = Path(os.environ.get("TMPDIR", "/tmp")) / f"lbm_clocks_{os.getpid()}.csv"

    def __enter__(self):
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}", f"--query-gpu={q}", "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=self.f, stderr=subprocess.DEVNULL,
            )
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if not self.path.exists():
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for name, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        self.path.unlink(missing_ok=True)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": smax, "reasons": sorted(reasons), "samples": len(sm)}


def barrier_max(value, world):
    from implexity_b200 import replicas

    return replicas.max_over_ranks(value) if world > 1 else value


def barrier(world):
    from implexity_b200 import replicas

    if world > 1:
        replicas.barrier()


def run_gpu(args, rank, world, local):
    import torch

    torch.cuda.set_device(local)
    from implexity_b200 import LbmSolver, normalize, workloads

    shape, T, coll = CONFIGS[args.config][:3]
    variants = [v for v in args.variants.split(",") if v]
    results = {}
    hbm, peak_kind = peaks()
    for variant in variants:
        storage = "float16" if variant == "fp16" else "float32"
        prob = workloads.config_problem(args.config, storage=storage)
        norm = normalize(prob)
        raw = workloads.config_design(args.config, 0)
        raw_pinned = torch.from_numpy(raw).pin_memory().numpy()
        w = workloads.objective_weights()
        s = LbmSolver(norm)
        cells = s.cells
        fwd_b = FWD_BYTES[(storage, s.q)]
        lam_storage = storage
        adj_b = adj_bytes(s.q, 2 if lam_storage == "float16" else 4)

        def iteration():
            s.set_design(raw_pinned)
            d = s.forward()
            r = s.responses()
            g, rep = s.gradient(w, mode="steady", tolerance=1e-8, lambda_storage=lam_storage, check_every=100)
            return d, r, g, rep

        for _ in range(args.warmup):
            iteration()
        barrier(world)
        torch.cuda.synchronize()
        fwd_ms = adj_ms = sens_ms = 0.0
        iters = 0
        wall = 0.0
        with Clocks(local) as clk:
            for _ in range(args.steps):
                t0 = time.perf_counter()
                d, r, g, rep = iteration()
                wall += time.perf_counter() - t0
                fwd_ms += d.device_ms
                adj_ms += rep.adjoint_ms
                sens_ms += rep.sensitivity_ms
                iters += rep.iterations
        torch.cuda.synchronize()
        barrier(world)
        dev_s = barrier_max((fwd_ms + adj_ms + sens_ms) / 1e3, world)
        wall = barrier_max(wall, world)
        lups = cells * (T * args.steps + iters)
        value = world * lups / dev_s / 1e6
        e2e = world * lups / wall / 1e6
        grid_tag = f"{shape[0]}x{shape[1]}x{shape[2]}"

        def roof(kind, lups, ms, bytes_cell):
            """Roofline of one stepping kernel: algorithmic bytes per cell update x
            cell updates / its device time (CUDA events), against the measured peak."""
            tag = f"k_{kind}_d3q{s.q}_{coll}_{storage}_{grid_tag}"
            achieved = lups / (ms / 1e3) * bytes_cell / 1e9 if ms > 0 else None
            traffic_cell = profiled_traffic(tag)
            return {
                "bound": "hbm",
                "achieved": achieved,
                "peak": hbm,
                "unit": "GB/s",
                "frac": None if achieved is None else achieved / hbm,
                "traffic": None if traffic_cell is None else traffic_cell * cells,
                "peak_kind": peak_kind,
                "kernel": tag,
                "bytes_per_cell": bytes_cell,
                "device_ms_per_step": ms / args.steps,
            }

        fwd_roof = roof("forward", cells * T * args.steps, fwd_ms, fwd_b)
        adj_roof = roof("adjoint", cells * iters, adj_ms, adj_b)
        results[variant] = {
            "value": value,
            "e2e": e2e,
            "ms_per_step": dev_s * 1e3 / args.steps,
            "wall_ms_per_step": wall * 1e3 / args.steps,
            "forward_mlups": cells * T * args.steps / (fwd_ms / 1e3) / 1e6,
            "adjoint_mlups": cells * iters / (adj_ms / 1e3) / 1e6 if adj_ms > 0 else None,
            "adjoint_iterations_per_step": iters / args.steps,
            "adjoint_residual": rep.residual,
            # the dominant kernel of the iteration (most device time) carries the roofline
            "roofline": adj_roof if adj_ms > fwd_ms else fwd_roof,
            "forward_roofline": fwd_roof,
            "adjoint_roofline": adj_roof,
            "h2d_bytes_per_step": raw.size * 8,
            "d2h_bytes_per_step": raw.size * 8 + 8 * 8,
            "launches_per_step": 1 + 1 + T + 1 + 1 + 2 + iters / args.steps + 2,
            "clocks": clk.summary(),
            "responses": [float(x) for x in r],
        }
        s.close()
    return results


def run_profile_case(args):
    """A short case of the bench kernels for ncu: forward steps and adjoint
    iterations of the bench workload, no timing."""
    import torch

    from implexity_b200 import ConvergenceError, LbmSolver, normalize, workloads

    torch.cuda.set_device(0)
    storage = "float16" if args.variants.split(",")[0] == "fp16" else "float32"
    prob = workloads.config_problem(args.config, storage=storage, steps=args.forward_steps)
    s = LbmSolver(normalize(prob))
    raw = workloads.config_design(args.config, 0)
    s.set_design(raw)
    d = s.forward()
    try:
        s.gradient(workloads.objective_weights(), mode="steady", tolerance=1e-30, lambda_storage=storage,
                   max_iterations=args.adjoint_iterations, check_every=args.adjoint_iterations)
    except ConvergenceError:
        pass
    print(json.dumps({"profile_case": args.config, "storage": storage, "forward_steps": args.forward_steps,
                      "adjoint_iterations": args.adjoint_iterations, "forward_ms": d.device_ms}))


def cpu_sample(config, seconds_target=15.0, threads=None):
    """Oracle (FP64 CPU) forward + transposed steps on the same workload."""
    from implexity_b200 import normalize, workloads
    from oracle import oracle as orc

    if threads:
        orc.set_threads(threads)
    prob = workloads.config_problem(config)
    norm = normalize(prob)
    o = orc.Oracle(norm)
    raw = workloads.config_design(config, 0)
    phi, alpha = o.design(raw)
    f = o.initial()
    lam = np.random.default_rng(0).standard_normal(f.shape) * 1e-3
    n = 0
    t0 = time.perf_counter()
    while True:
        f, _ = o.interval(f, alpha)
        lam, _ = o.interval_vjp(f, alpha, lam)
        n += 1
        if time.perf_counter() - t0 > seconds_target and n >= 2:
            break
    el = time.perf_counter() - t0
    lups = 2 * n * o.cells
    return {
        "value": lups / el / 1e6,
        "unit": "MLUPS",
        "cores": orc.threads(),
        "kind": "port",
        "sample": f"{n} forward steps + {n} transposed steps of the {config} workload ({o.cells} cells), FP64, "
                  f"{el:.1f} s",
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="native", choices=["native", "reference"])
    ap.add_argument("--config", default="channel256x128x128_trt", choices=sorted(CONFIGS))
    ap.add_argument("--variants", default="fp32,fp16")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--profile", action="store_true", help="run a short case of the bench kernels for ncu")
    ap.add_argument("--forward-steps", type=int, default=20)
    ap.add_argument("--adjoint-iterations", type=int, default=20)
    args = ap.parse_args()
    if args.profile:
        run_profile_case(args)
        return
    rank, world, local = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1")), 0
    metric = "MLUPS fwd+adjoint D3Q19, FP32 vs FP16-store at grad err<1e-3; % HBM roofline"
    shape, T, coll, bulk, _ = CONFIGS[args.config]
    config = {
        "workload": f"{args.config}: D3Q19 {coll.upper()} {shape[0]}x{shape[1]}x{shape[2]} channel, {T} forward "
                    f"steps + steady adjoint to 1e-8 + design-map transpose per step",
        "cells": int(np.prod(shape)),
        "forward_steps": T,
        "l2": "populations (>=80 MB) larger than L2 on every step; no flush",
        "parallelism": f"replicas{args.gpus}" if args.gpus > 1 else "single",
    }
    if args.impl == "reference":
        if rank != 0:
            return
        vals = []
        for _ in range(args.warmup):
            cpu_sample(args.config, seconds_target=min(args.cpu_seconds, 5.0))
        for _ in range(args.steps):
            vals.append(cpu_sample(args.config, seconds_target=args.cpu_seconds))
        v = float(np.mean([x["value"] for x in vals]))
        line = {
            "metric": metric, "value": v, "unit": "MLUPS", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": None, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config, "impl": "reference",
            "cpu_baseline": {**vals[-1], "value": v},
            "e2e": {"value": v, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        }
        print(json.dumps(line))
        return
    from implexity_b200 import replicas

    rank, world, local = replicas.init("nccl")
    res = run_gpu(args, rank, world, local)
    cpu = None
    if rank == 0 and world == 1:
        cpu = cpu_sample(args.config, seconds_target=args.cpu_seconds)
    replicas.finalize()
    if rank != 0:
        return
    head = res.get("fp32") or next(iter(res.values()))
    line = {
        "metric": metric,
        "value": head["value"],
        "unit": "MLUPS",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": head["ms_per_step"],
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic",
        "config": config,
        "e2e": {"value": head["e2e"], "unit": "MLUPS", "h2d_bytes_per_step": head["h2d_bytes_per_step"],
                "d2h_bytes_per_step": head["d2h_bytes_per_step"]},
        "gpu_launches": int(round(head["launches_per_step"] * args.steps)),
        "roofline": head["roofline"],
        "cpu_baseline": cpu,
        "clocks": head["clocks"],
        "variants": {k: {kk: vv for kk, vv in v.items() if kk not in ("clocks",)} for k, v in res.items()},
    }
    if "fp16" in res and "fp32" in res:
        line["fp16_speedup"] = res["fp16"]["value"] / res["fp32"]["value"]
    print(json.dumps(line))


if __name__ == "__main__":
    main()
