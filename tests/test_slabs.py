"""x-slab domain decomposition (implexity_b200.slabs) on CPU: the partition,
the halo plan, and two gloo ranks running the decomposed forward trajectory,
admission, responses and steady adjoint through the slab driver over the FP64
oracle's cell-range pieces (tests/_slab_oracle.py) -- against the
single-domain oracle.  Arrays hold NaN outside each rank's cells and the halo
slots the plan delivers, so a missing halo slot shows as NaN."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

from implexity_b200 import slabs


def test_partition_covers_the_grid():
    for nx, world in [(16, 2), (17, 3), (64, 8), (9, 4)]:
        parts = slabs.partition(nx, world)
        assert parts[0].x_begin == 0 and parts[-1].x_end == nx
        assert all(a.x_end == b.x_begin for a, b in zip(parts, parts[1:]))
        sizes = [p.x_end - p.x_begin for p in parts]
        assert max(sizes) - min(sizes) <= 1 and min(sizes) >= 2
    with pytest.raises(ValueError):
        slabs.partition(5, 3)
    s = slabs.partition(10, 2, periodic_x=True)
    assert (s[0].left, s[0].right, s[1].left, s[1].right) == (1, 1, 0, 0)
    s = slabs.partition(10, 2)
    assert (s[0].left, s[1].right) == (None, None)


@pytest.mark.parametrize("q,ndir", [(19, 5), (27, 9)])
def test_halo_plan_carries_the_crossing_directions(q, ndir):
    plus, minus = slabs.crossing(q, +1), slabs.crossing(q, -1)
    assert len(plus) == len(minus) == ndir
    st = {m.side: m.directions for m in slabs.halo_plan(q, "state")}
    ad = {m.side: m.directions for m in slabs.halo_plan(q, "adjoint")}
    assert st == {"right": tuple(plus), "left": tuple(minus)}
    assert ad == {"right": tuple(minus), "left": tuple(plus)}


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _case(name):
    from implexity_b200 import workloads

    if name == "channel":
        prob = workloads.channel_problem(shape=(16, 8, 6), steps=60, collision="trt")
        solid = np.zeros((16, 8, 6), bool)
        solid[7:9, 3:5, 1:3] = True  # straddles the slab boundary at x = 8
        prob["solid_mask"] = solid
        prob["design_region"] = np.asarray(prob["design_region"]) & ~solid
        return prob
    if name == "periodic_d3q27":
        prob = workloads.channel_problem(shape=(12, 7, 6), steps=50, collision="trt", lattice="D3Q27", ports=False)
        prob["periodic_axes"] = [True, False, True]
        prob["acceleration_m_s2"] = [2e-5, 0.0, 0.0]
        prob["design_region"] = np.ones((12, 7, 6), bool)
        return prob
    raise ValueError(name)


def _worker(rank, world, port, name, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port), OMP_NUM_THREADS="2")
    import sys
    from pathlib import Path

    sys.path.insert(0, str(Path(__file__).resolve().parent))
    from implexity_b200 import normalize, replicas, workloads
    from _slab_oracle import OracleSlab

    replicas.init("gloo", timeout_s=60)
    prob = _case(name)
    norm = normalize(prob)
    raw = workloads.uniform_design(norm.shape, 3)
    part = slabs.partition(norm.shape[0], world, periodic_x=bool(norm.periodic_axes[0]))
    backend = OracleSlab(norm, part[rank], raw)
    drv = slabs.SlabDriver(backend, slabs.TorchComm(), mach_limit=norm.mach_limit)
    adm = drv.forward(norm.step_count)
    r = drv.responses()
    res = {"admission": {k: v for k, v in adm.items() if k not in ("mass", "exchange")},
           "mass": np.asarray(adm["mass"]), "exchange": np.asarray(adm["exchange"]),
           "state": backend.final_state(), "responses": r}
    if norm.ports:  # a closed periodic box conserves mass: its steady adjoint has no fixed point
        g, rep = drv.gradient_steady(workloads.objective_weights(), tolerance=1e-10, check_every=20)
        res.update(grad=g, converged=rep["converged"])
    out[rank] = res
    replicas.finalize()


@pytest.mark.parametrize("name", ["channel", "periodic_d3q27"])
def test_two_slabs_reproduce_the_single_domain_oracle(name):
    from implexity_b200 import normalize, workloads
    from oracle.oracle import Oracle

    world = 2
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, name, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    res = dict(out)

    norm = normalize(_case(name))
    o = Oracle(norm)
    raw = workloads.uniform_design(norm.shape, 3)
    phi, alpha = o.design(raw)
    f_ref, d_ref, mass_ref, exch_ref = o.history_trace(alpha, norm.step_count)
    state = np.concatenate([res[r]["state"] for r in range(world)])
    assert np.all(np.isfinite(state))
    np.testing.assert_allclose(state, f_ref, rtol=0, atol=1e-13)
    for r in range(world):
        np.testing.assert_allclose(res[r]["mass"], mass_ref, rtol=1e-13)
        np.testing.assert_allclose(res[r]["exchange"][1:], exch_ref[1:], rtol=1e-9, atol=1e-13)
        a = res[r]["admission"]
        assert a["admitted"] == bool(d_ref.admitted)
        assert abs(a["maximum_mach"] - d_ref.maximum_mach) <= 1e-12
        assert abs(a["relative_mass_drift"] - d_ref.relative_mass_drift) <= 1e-12
        r_ref = o.vector(phi, alpha, f_ref)
        np.testing.assert_allclose(res[r]["responses"], r_ref, rtol=1e-10, atol=1e-12 * np.max(np.abs(r_ref)))
    if not norm.ports:
        return
    w = workloads.objective_weights()
    g_ref, _, _, st = o.gradient(raw, w, mode="steady", tol=1e-12)
    assert st == 0
    for r in range(world):
        assert res[r]["converged"]
        err = np.linalg.norm(res[r]["grad"] - g_ref) / np.linalg.norm(g_ref)
        assert err < 1e-8, err
