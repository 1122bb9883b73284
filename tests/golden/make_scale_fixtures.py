"""Generates the FP64 fixtures of the oracle-grid parity checks
(tests/test_scale_parity.py) and of the finite-difference check at the
specified step (tests/test_fd_fixture.py) by running the FP64 CPU oracle
(oracle/, test infrastructure) once.  The GPU tests then compare against the
stored numbers in seconds instead of re-running the oracle for minutes.

Cases (all seeded; the designs are regenerated from their seeds by the tests):

  scale_channel64_trt   the 64^3 oracle grid of the 128^3 channel workload:
                        D3Q19 TRT (tau 0.8, magic 3/16), plug inlet 0.05,
                        box filter, 5000 steps, steady adjoint (Neumann
                        series, implicit.rs:49-67 semantics) to 1e-12.
  scale_spheres_mrt     the MRT sphere workload reduced to 64x32x32 (shear
                        rate 1.0, bulk rate 1.2, 20 spheres with radii scaled
                        to the grid, blended 0.3 with noise), inlet 0.03,
                        3000 steps, steady adjoint to 1e-12.
  fd_channel32_trt      central differences (gradcheck.rs:218-232, taken
                        along a direction) at step 1e-4 along 8 seeded
                        Gaussian directions (seeds 0..7, implexity_b200.
                        gradcheck.directions) of J = pressure drop + viscous
                        dissipation after 5000 steps of the 32^3 channel,
                        with the FP64 oracle as the forward; plus the
                        oracle's horizon and steady directional derivatives.

Stored per field case: the eight responses (FP64), rho - 1 and the
Brinkman-corrected velocity of the final state and the steady gradient
(FP32: their rounding, ~6e-8 relative, is far below the 1e-5 / 1e-4 bars).

Run: python tests/golden/make_scale_fixtures.py [case ...]   (minutes, all host threads)
"""
from __future__ import annotations

import sys
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent.parent
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(HERE.parent))

from implexity_b200 import normalize, workloads  # noqa: E402
from implexity_b200.gradcheck import directions  # noqa: E402
from oracle.oracle import Oracle  # noqa: E402

FD_STEP = 1e-4
FD_DIRECTIONS = 8


def fields(o, f, alpha):
    from test_gpu_parity import macroscopic

    rho, u = macroscopic(f, o.q, alpha, o.acceleration_lattice)
    return (rho - 1.0).astype(np.float32), u.T.astype(np.float32).copy()


def field_case(norm, raw, tol=1e-12):
    o = Oracle(norm)
    w = workloads.objective_weights()
    t0 = time.perf_counter()
    g, r, rep, st = o.gradient(raw, w, mode="steady", tol=tol)
    assert st == 0, "oracle steady adjoint did not converge"
    _, alpha = o.design(raw)
    f, d = o.history(alpha, norm.step_count)
    assert d.admitted
    rho1, u = fields(o, f, alpha)
    print(f"  {time.perf_counter() - t0:.0f} s, {rep.iterations} adjoint iterations, residual {rep.residual:.2e}")
    return {
        "responses": r,
        "rho_minus_1": rho1,
        "u": u,
        "grad_steady": g.astype(np.float32),
        "adjoint_iterations": np.int64(rep.iterations),
        "adjoint_tolerance": np.float64(tol),
        "maximum_mach": np.float64(d.maximum_mach),
    }


def scale_channel64_trt():
    shape, steps, coll, _, _ = workloads.CONFIGS["channel64_trt"]
    norm = normalize(workloads.channel_problem(shape=shape, steps=steps, collision=coll))
    out = field_case(norm, workloads.uniform_design(shape, 0))
    out.update(shape=np.array(shape), steps=np.int64(steps), design_seed=np.int64(0))
    return out


SPHERES = {"name": "channel256x128x128_mrt", "shape": (64, 32, 32), "steps": 3000, "u_in": 0.03}


def spheres_problem(storage="float32"):
    s = SPHERES
    return workloads.config_problem(s["name"], storage=storage, steps=s["steps"], shape=s["shape"], u_in=s["u_in"])


def scale_spheres_mrt():
    s = SPHERES
    norm = normalize(spheres_problem())
    out = field_case(norm, workloads.config_design(s["name"], 0, shape=s["shape"]))
    out.update(shape=np.array(s["shape"]), steps=np.int64(s["steps"]), design_seed=np.int64(0))
    return out


FD = {"shape": (32, 32, 32), "steps": 5000, "design_seed": 2}


def fd_problem(storage="float32"):
    return workloads.channel_problem(shape=FD["shape"], steps=FD["steps"], collision="trt", storage=storage)


def fd_channel32_trt():
    norm = normalize(fd_problem())
    o = Oracle(norm)
    w = workloads.objective_weights()
    shape = FD["shape"]
    raw = workloads.uniform_design(shape, FD["design_seed"])
    editable = (np.asarray(norm.design_region, bool) & ~np.asarray(norm.solid_mask, bool)).reshape(shape)

    def J(x):
        phi, alpha = o.design(x)
        f, d = o.history(alpha, FD["steps"])
        assert d.admitted
        return float(np.dot(w, o.vector(phi, alpha, f)))

    t0 = time.perf_counter()
    g_h, r0, _, st = o.gradient(raw, w, mode="horizon", K=100)
    assert st == 0
    g_s, _, rep_s, st = o.gradient(raw, w, mode="steady", tol=1e-12)
    assert st == 0
    seeds, fd, ad_h, ad_s = [], [], [], []
    for s, d in directions(raw, editable, FD_DIRECTIONS, 0, FD_STEP):
        jp, jm = J(raw + FD_STEP * d), J(raw - FD_STEP * d)
        seeds.append(s)
        fd.append((jp - jm) / (2.0 * FD_STEP))
        ad_h.append(float(np.dot(g_h, d.ravel())))
        ad_s.append(float(np.dot(g_s, d.ravel())))
        print(f"  direction {s}: fd {fd[-1]:.10e} horizon {ad_h[-1]:.10e} steady {ad_s[-1]:.10e}", flush=True)
    print(f"  {time.perf_counter() - t0:.0f} s")
    return {
        "shape": np.array(shape),
        "steps": np.int64(FD["steps"]),
        "design_seed": np.int64(FD["design_seed"]),
        "fd_step": np.float64(FD_STEP),
        "seeds": np.array(seeds),
        "fd": np.array(fd),
        "oracle_horizon": np.array(ad_h),
        "oracle_steady": np.array(ad_s),
        "objective": np.float64(np.dot(w, r0)),
        "responses": r0,
    }


CASES = {
    "scale_channel64_trt": scale_channel64_trt,
    "scale_spheres_mrt": scale_spheres_mrt,
    "fd_channel32_trt": fd_channel32_trt,
}


def main(names):
    for name in names or CASES:
        print(name, flush=True)
        np.savez_compressed(HERE / f"{name}.npz", **CASES[name]())


if __name__ == "__main__":
    main(sys.argv[1:])
