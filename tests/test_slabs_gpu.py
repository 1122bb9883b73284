"""x-slab decomposition through the CUDA library on one GPU: two slab handles
(lbm_create_slab) driven by two host threads, their halos handed over through
device buffers (no kernel waits on another: the threads exchange between
launches), against one single-domain handle of the same problem.

Bars: the owned cells' final populations, the admission record and the
responses within 1e-6 relative (FP32 with a different summation order), the
steady gradient within 1e-5 relative L2.
"""
import threading

import numpy as np
import pytest

from implexity_b200 import LbmSolver, normalize, slabs, workloads
from implexity_b200.slab_solver import SlabSolver

pytestmark = pytest.mark.gpu


class ThreadComm:
    """Ranks as threads of one process: halos are handed over by reference."""

    def __init__(self, world):
        self.world = world
        self.bar = threading.Barrier(world, timeout=60)
        self.box = [None] * world

    def view(self, rank):
        comm = self

        class View:
            def __init__(self):
                self.rank, self.world = rank, comm.world

            def exchange(self, sends, recv_like, peers):
                comm.box[rank] = sends
                comm.bar.wait()
                mirror = {"left": "right", "right": "left"}
                out = {side: comm.box[peer][mirror[side]] for side, peer in peers.items() if peer is not None}
                comm.bar.wait()
                return out

            def allreduce(self, values, op="sum"):
                comm.box[rank] = np.asarray(values, dtype=np.float64)
                comm.bar.wait()
                stack = np.stack([comm.box[r] for r in range(comm.world)])
                comm.bar.wait()
                return {"sum": stack.sum(0), "min": stack.min(0), "max": stack.max(0)}[op]

        return View()


def _channel():
    shape = (24, 10, 8)
    solid = np.zeros(shape, bool)
    solid[11:13, 4:7, 2:5] = True  # straddles the slab boundary at x = 12
    prob = workloads.channel_problem(shape=shape, steps=150, collision="trt", box_half_width=0,
                                     filter_radius_cells=2.0, solid=solid)
    return prob


def _periodic():
    shape = (16, 7, 6)
    prob = workloads.channel_problem(shape=shape, steps=100, collision="trt", lattice="D3Q27", ports=False)
    prob["periodic_axes"] = [True, False, True]
    prob["acceleration_m_s2"] = [2e-5, 0.0, 0.0]
    prob["design_region"] = np.ones(shape, bool)
    return prob


def _run_slabs(prob, raw, world, halo, gradient):
    norm = normalize(prob)
    part = slabs.partition(norm.shape[0], world, periodic_x=bool(norm.periodic_axes[0]))
    comm = ThreadComm(world)
    out, errors = [None] * world, []

    def rank_main(r):
        try:
            b = SlabSolver(norm, part[r], halo=halo)
            b.set_design(raw)
            drv = slabs.SlabDriver(b, comm.view(r), mach_limit=norm.mach_limit)
            res = {"admission": drv.forward(norm.step_count), "responses": drv.responses()}
            res["state"] = b.populations()[b.owned_cells()]
            if gradient:
                res["grad"], res["report"] = drv.gradient_steady(workloads.objective_weights(), tolerance=1e-10,
                                                                 check_every=20)
            out[r] = res
            b.close()
        except Exception as e:  # noqa: BLE001  (reported by the main thread)
            errors.append(e)
            comm.bar.abort()

    threads = [threading.Thread(target=rank_main, args=(r,)) for r in range(world)]
    for t in threads:
        t.start()
    for t in threads:
        t.join(timeout=300)
    if errors:
        raise errors[0]
    return norm, out


@pytest.mark.parametrize("case", ["channel", "periodic_d3q27"])
def test_two_slab_handles_match_one_handle(gpu_lib, case):
    prob = _channel() if case == "channel" else _periodic()
    raw = workloads.uniform_design(tuple(prob["shape"]), 5)
    gradient = case == "channel"  # a closed periodic box has no steady adjoint fixed point
    norm, res = _run_slabs(prob, raw, world=2, halo=2, gradient=gradient)
    with LbmSolver(norm) as s:
        s.set_design(raw)
        d = s.forward()
        f = s.populations()
        r_ref = s.responses()
        traj = s.trajectory()
        g_ref = s.gradient(workloads.objective_weights(), mode="steady", tolerance=1e-10)[0] if gradient else None
    state = np.concatenate([res[r]["state"] for r in range(2)])
    assert float(np.max(np.abs(state - f)) / np.max(np.abs(f))) < 1e-6
    for r in range(2):
        a = res[r]["admission"]
        assert a["admitted"] == d.admitted
        np.testing.assert_allclose(a["mass"], traj["mass"], rtol=1e-9)
        assert abs(a["maximum_mach"] - d.maximum_mach) <= 1e-6 * d.maximum_mach
        np.testing.assert_allclose(res[r]["responses"], r_ref, rtol=1e-6, atol=1e-6 * np.max(np.abs(r_ref)))
        if gradient:
            assert res[r]["report"]["converged"]
            g = res[r]["grad"].reshape(g_ref.shape)
            assert float(np.linalg.norm(g - g_ref) / np.linalg.norm(g_ref)) < 1e-5
