"""Seeded synthetic problems with the shapes and parameters of the benchmark
configurations (no dataset is involved: every input is generated here).

The channel: plug velocity inlet at x = 0 (interior face cells; the y/z edge
cells are excluded because ports may not touch closed faces, ports.rs:185-197),
constant-density outlet at x = nx-1, halfway bounce-back walls on y and z, a
porous design region between the port planes, RAMP resistance
alpha = dt * drag_max * q (1 - phi) / (q + phi) with dt * drag_max = 0.1 and
q = 0.1 (alpha in [0, 0.1]).  Physical units: dx = 1 mm, water viscosity, the
time step chosen for the requested relaxation time.
"""
from __future__ import annotations

import numpy as np

NU = 1e-6
DX = 1e-3


# The seeded channel workloads: name -> (shape, forward steps, collision,
# MRT bulk rate, design kind).
CONFIGS = {
    "channel128_trt": ((128, 128, 128), 5000, "trt", None, "uniform"),
    "channel256x128x128_trt": ((256, 128, 128), 3000, "trt", None, "uniform"),
    "channel256x128x128_mrt": ((256, 128, 128), 3000, "mrt", 1.2, "spheres"),
    "channel48x24x24_trt": ((48, 24, 24), 2000, "trt", None, "uniform"),
    "channel64_trt": ((64, 64, 64), 5000, "trt", None, "uniform"),
}
# Relaxation time where it is not the channel's 0.8: the MRT sphere workload
# relaxes shear at rate 1.0 (tau = 1) and bulk at 1.2.
CONFIG_TAU = {"channel256x128x128_mrt": 1.0}
# The unsteady D3Q27 workload: shape, steps, inlet period in steps.
PULSATILE = {"pulsatile192_d3q27": ((192, 192, 192), 4000, 1000)}


def config_problem(name: str, storage: str = "float32", steps: int | None = None, shape=None, **kw) -> dict:
    """The problem of a named workload (optionally with another step count,
    grid shape or channel_problem keyword, for reduced-size checks)."""
    shp, T, coll, bulk, _ = CONFIGS[name]
    return channel_problem(shape=tuple(shape) if shape is not None else shp, steps=T if steps is None else steps,
                           collision=coll, storage=storage, mrt_bulk_rate=bulk, tau=CONFIG_TAU.get(name, 0.8), **kw)


def config_design(name: str, seed: int = 0, shape=None) -> np.ndarray:
    """The seeded raw design of a named workload.  On another grid shape the
    sphere radii scale with the grid, so the blocked volume stays the same."""
    full, _, _, _, kind = CONFIGS[name]
    shp = tuple(shape) if shape is not None else full
    if kind == "uniform":
        return uniform_design(shp, seed)
    f = shp[0] / full[0]
    return sphere_design(shp, seed, rmin=4.0 * f, rmax=12.0 * f)


def channel_problem(
    shape=(48, 24, 24),
    steps=2000,
    tau=0.8,
    u_in=0.05,
    collision="trt",
    lattice="D3Q19",
    storage="float32",
    box_half_width=1,
    filter_radius_cells=0.0,
    mrt_bulk_rate=None,
    adjoint=None,
    mach_limit=0.2,
    ports=True,
    solid=None,
):
    nx, ny, nz = shape
    dt = (tau - 0.5) / 3.0 * DX * DX / NU
    vel = u_in * DX / dt
    n = nx * ny * nz
    solid_mask = np.zeros(shape, dtype=bool) if solid is None else np.asarray(solid, dtype=bool)
    design = np.zeros(shape, dtype=bool)
    design[1 : nx - 1] = True
    design &= ~solid_mask
    fixed = np.ones(shape)
    port_list = []
    if ports:
        inlet = np.zeros(shape, dtype=bool)
        inlet[0, 1 : ny - 1, 1 : nz - 1] = True
        outlet = np.zeros(shape, dtype=bool)
        outlet[nx - 1, 1 : ny - 1, 1 : nz - 1] = True
        port_list = [
            {"id": "inlet", "kind": "velocity", "face": "xmin", "mask": inlet, "velocity_m_s": [vel, 0.0, 0.0]},
            {
                "id": "outlet",
                "kind": "pressure",
                "face": "xmax",
                "mask": outlet,
                "velocity_m_s": [0.0, 0.0, 0.0],
                "gauge_pressure_Pa": 0.0,
            },
        ]
    coll = {"kind": collision}
    if collision == "trt":
        coll["magic"] = 3.0 / 16.0
    if collision == "mrt":
        coll["odd_magic"] = 3.0 / 16.0
        coll["bulk_rate"] = mrt_bulk_rate
    opts = {"lattice": lattice, "collision": coll, "population_storage": storage}
    if box_half_width:
        opts["filter"] = {"kind": "box", "half_width": int(box_half_width)}
    if adjoint:
        opts["adjoint"] = adjoint
    problem = {
        "shape": list(shape),
        "spacing_m": DX,
        "step_s": dt,
        "step_count": int(steps),
        "density_kg_m3": 1000.0,
        "kinematic_viscosity_m2_s": NU,
        "acceleration_m_s2": [0.0, 0.0, 0.0],
        "periodic_axes": [False, False, False],
        "solid_mask": solid_mask,
        "design_region": design,
        "fixed_design": fixed,
        "drag_max_per_s": 0.1 / dt,
        "drag_shape": 0.1,
        "mach_limit": mach_limit,
        "history_byte_budget": (int(steps) + 1) * n * 19 * 8,
        "topology_map": {"filter_radius_m": filter_radius_cells * DX, "projection_beta": 0.0, "projection_eta": 0.5},
        "ports": port_list,
        "solver_options": opts,
    }
    return problem


def pulsatile_problem(shape=(192, 192, 192), steps=4000, lattice="D3Q27", tau=0.8, u_mean=0.04, amp_frac=0.5,
                      period_steps=1000, ramp_steps=0, storage="float32", box_half_width=1):
    """The unsteady channel: the plug inlet pulses as u(t) = u_mean (1 + amp_frac
    sin(2 pi t / (period_steps dt))) (lattice units), optionally ramped in over
    ramp_steps; the objective is the time average of the responses (solver
    option time_average)."""
    prob = channel_problem(shape=shape, steps=steps, tau=tau, u_in=u_mean, collision="trt", lattice=lattice,
                           storage=storage, box_half_width=box_half_width)
    dt = prob["step_s"]
    inlet = prob["ports"][0]
    inlet["amplitude_m_s"] = [amp_frac * inlet["velocity_m_s"][0], 0.0, 0.0]
    inlet["frequency_hz"] = 1.0 / (period_steps * dt)
    inlet["phase_rad"] = 0.0
    inlet["ramp_s"] = ramp_steps * dt
    prob["solver_options"]["time_average"] = True
    return prob


def uniform_design(shape, seed=0):
    return np.random.default_rng(seed).uniform(0.0, 1.0, size=shape)


def sphere_design(shape, seed=0, n_spheres=20, rmin=4.0, rmax=12.0, blend=0.3):
    """Union of solid spheres (raw 0 inside) blended with uniform noise."""
    rng = np.random.default_rng(seed)
    nx, ny, nz = shape
    inside = np.zeros(shape, dtype=bool)
    I, J, K = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    for _ in range(n_spheres):
        r = rng.uniform(rmin, rmax)
        c = rng.uniform([0, 0, 0], [nx, ny, nz])
        inside |= (I - c[0]) ** 2 + (J - c[1]) ** 2 + (K - c[2]) ** 2 <= r * r
    noise = rng.uniform(0.0, 1.0, size=shape)
    return (1.0 - blend) * (~inside) + blend * noise


def objective_weights():
    """J = inlet-outlet pressure drop [Pa] + total viscous dissipation [W]."""
    w = np.zeros(8)
    w[6] = 1.0
    w[7] = 1.0
    return w
