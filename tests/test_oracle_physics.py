"""Known-answer physics for the FP64 oracle (the reference ships no LBM
tests; these pin the restatement to analytic solutions):

* body-force Poiseuille flow between halfway bounce-back walls: TRT with magic
  3/16 puts the wall exactly half a link out for any tau (moving/options.rs:
  53-55), so the parabola is reproduced to rounding;
* uniform Brinkman medium: steady velocity a / alpha exactly;
* MRT with default rates reproduces TRT (moving/options.rs:56-58);
* closed periodic box without ports conserves mass to rounding.
"""
import numpy as np
import pytest

from implexity_b200 import normalize
from oracle.oracle import Oracle, mrt_basis

from _problems import golden_problem  # noqa: F401  (puts tests/golden on the path)


def box_problem(shape, coll="trt", lattice="D3Q19", tau=0.8, accel=(1e-6, 0, 0), periodic=(True, False, True),
                raw_design=False, bulk=None):
    dx, nu = 1e-3, 1e-6
    dt = (tau - 0.5) / 3 * dx * dx / nu
    n = int(np.prod(shape))
    coll_opts = {"kind": coll}
    if coll == "mrt":
        coll_opts["bulk_rate"] = bulk
    return {
        "shape": list(shape), "spacing_m": dx, "step_s": dt, "step_count": 10,
        "density_kg_m3": 1000.0, "kinematic_viscosity_m2_s": nu,
        "acceleration_m_s2": list(accel), "periodic_axes": list(periodic),
        "solid_mask": np.zeros(shape, bool), "design_region": np.full(shape, raw_design),
        "fixed_design": np.ones(shape), "drag_max_per_s": 0.1 / dt, "drag_shape": 0.1, "mach_limit": 0.2,
        "history_byte_budget": 11 * n * 19 * 8,
        "solver_options": {"lattice": lattice, "collision": coll_opts},
    }


def velocity(o, f, alpha, q):
    from test_gpu_parity import macroscopic  # same helper as the GPU tests

    return macroscopic(f, q, alpha, o.acceleration_lattice)


@pytest.mark.parametrize("lattice", ["D3Q19", "D3Q27"])
@pytest.mark.parametrize("tau", [0.6, 0.8, 1.5])
def test_trt_poiseuille_is_exact(lattice, tau):
    ny = 8
    p = box_problem((2, ny, 2), "trt", lattice, tau)
    o = Oracle(normalize(p))
    alpha = np.zeros(o.cells)
    steps = int(40 * ny * ny / ((tau - 0.5) / 3))
    f, d = o.history(alpha, steps)
    _, u = velocity(o, f, alpha, o.q)
    a = o.acceleration_lattice[0]
    nu = (o.tau - 0.5) / 3
    y = np.arange(ny) + 0.5
    exact = a / (2 * nu) * y * (ny - y)
    ux = u[:, 0].reshape(2, ny, 2)[0, :, 0]
    np.testing.assert_allclose(ux, exact, rtol=1e-9)
    assert d.relative_mass_drift < 1e-11


def test_bgk_poiseuille_wall_slip_depends_on_tau():
    ny = 8
    errs = []
    for tau in (0.6, 1.9):
        p = box_problem((2, ny, 2), "bgk", "D3Q19", tau)
        o = Oracle(normalize(p))
        alpha = np.zeros(o.cells)
        f, _ = o.history(alpha, int(40 * ny * ny / ((tau - 0.5) / 3)))
        _, u = velocity(o, f, alpha, 19)
        a, nu = o.acceleration_lattice[0], (o.tau - 0.5) / 3
        y = np.arange(ny) + 0.5
        exact = a / (2 * nu) * y * (ny - y)
        errs.append(np.max(np.abs(u[:, 0].reshape(2, ny, 2)[0, :, 0] - exact) / exact.max()))
    assert errs[0] < 5e-2 and errs[1] > 5 * errs[0]


@pytest.mark.parametrize("coll", ["bgk", "trt", "mrt"])
def test_uniform_brinkman_velocity(coll):
    p = box_problem((3, 3, 3), coll, "D3Q19", 0.8, accel=(2e-6, 1e-6, 0), periodic=(True, True, True), raw_design=True,
                    bulk=1.2 if coll == "mrt" else None)
    o = Oracle(normalize(p))
    phi, alpha = o.design(np.full(27, 0.3))
    f, _ = o.history(alpha, 3000)
    _, u = velocity(o, f, alpha, 19)
    a = np.asarray(o.acceleration_lattice)
    np.testing.assert_allclose(u, np.tile(a / alpha[0], (27, 1)), rtol=1e-10, atol=1e-15)


@pytest.mark.parametrize("lattice", ["D3Q19", "D3Q27"])
def test_mrt_default_rates_reproduce_trt(lattice):
    p_trt = box_problem((6, 5, 4), "trt", lattice, 0.9, periodic=(True, False, False), raw_design=True)
    p_mrt = box_problem((6, 5, 4), "mrt", lattice, 0.9, periodic=(True, False, False), raw_design=True)
    raw = np.random.default_rng(3).uniform(0, 1, 120)
    out = []
    for p in (p_trt, p_mrt):
        o = Oracle(normalize(p))
        _, alpha = o.design(raw)
        out.append(o.history(alpha, 200)[0])
    np.testing.assert_allclose(out[1], out[0], rtol=0, atol=1e-15)


@pytest.mark.parametrize("q", [19, 27])
def test_mrt_basis_is_weighted_orthogonal(q):
    rows, norms, groups = mrt_basis(q)
    from test_gpu_parity import macroscopic  # noqa: F401

    if q == 19:
        c = np.array([[0, 0, 0], [-1, -1, 0], [-1, 0, -1], [-1, 0, 0], [-1, 0, 1], [-1, 1, 0], [0, -1, -1], [0, -1, 0],
                      [0, -1, 1], [0, 0, -1], [0, 0, 1], [0, 1, -1], [0, 1, 0], [0, 1, 1], [1, -1, 0], [1, 0, -1],
                      [1, 0, 0], [1, 0, 1], [1, 1, 0]])
    else:
        c = np.array([[0, 0, 0]] + [[a, b, d] for a in (-1, 0, 1) for b in (-1, 0, 1) for d in (-1, 0, 1)
                                    if (a, b, d) != (0, 0, 0)])
    n1 = (np.abs(c).sum(1))
    w = np.select([n1 == 0, n1 == 1, n1 == 2], [1 / 3, 1 / 18, 1 / 36], 0) if q == 19 else \
        np.select([n1 == 0, n1 == 1, n1 == 2, n1 == 3], [8 / 27, 2 / 27, 1 / 54, 1 / 216])
    G = rows @ np.diag(w) @ rows.T
    np.testing.assert_allclose(G, np.diag(norms), atol=1e-12)
    # odd groups (momentum, odd) span exactly the antisymmetric subspace
    opp = np.array([int(np.where((c == -c[i]).all(1))[0][0]) for i in range(q)])
    odd = np.isin(groups, [1, 4])
    assert odd.sum() == (q - 1) // 2
    np.testing.assert_allclose(rows[odd], -rows[odd][:, opp], atol=1e-12)
    np.testing.assert_allclose(rows[~odd], rows[~odd][:, opp], atol=1e-12)


def test_closed_box_conserves_mass():
    p = box_problem((6, 5, 4), "trt", "D3Q19", 0.7, periodic=(False, False, False), raw_design=True)
    o = Oracle(normalize(p))
    _, alpha = o.design(np.random.default_rng(1).uniform(0, 1, 120))
    _, d = o.history(alpha, 300)
    assert d.relative_mass_drift < 1e-13
    assert d.admitted
