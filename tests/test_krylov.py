"""The BiCGStab steady adjoint (lbm_adjoint_opts_t.steady_solver =
LBM_STEADY_BICGSTAB) against the Neumann series and the FP64 oracle.

Both solve (I - L) x = s for the transposed step L at the final state
(implicit.rs:49-67 semantics).  Bars: the two solvers' gradients agree within
1e-6 relative L2 when both are converged to 1e-10; BiCGStab's gradient meets
the oracle's steady gradient within 1e-4; on the 128^3 channel it needs at
least three times fewer operator applications than the Neumann series.
"""
import numpy as np
import pytest

from implexity_b200 import ContractError, LbmSolver, normalize, workloads
from oracle.oracle import Oracle
from test_gpu_parity import rel_l2

pytestmark = pytest.mark.gpu

CASES = [
    ("trt", "D3Q19", None),
    ("mrt", "D3Q27", None),
    ("trt", "D3Q19", "solid"),
]


def _problem(coll, lattice, solid_kind, shape=(24, 12, 10), steps=400):
    solid = None
    if solid_kind:
        solid = np.zeros(shape, bool)
        solid[8:11, 3:6, 0:4] = True  # touches the z wall
        solid[15:17, 8:12, 5:8] = True  # touches the y wall
    return workloads.channel_problem(shape=shape, steps=steps, collision=coll, lattice=lattice,
                                     mrt_bulk_rate=1.2 if coll == "mrt" else None, solid=solid)


@pytest.mark.parametrize("coll,lattice,solid_kind", CASES)
def test_bicgstab_matches_neumann_and_oracle(gpu_lib, coll, lattice, solid_kind):
    norm = normalize(_problem(coll, lattice, solid_kind))
    raw = workloads.uniform_design(norm.shape, 6)
    w = workloads.objective_weights()
    g_ref, _, _, st = Oracle(norm).gradient(raw, w, mode="steady", tol=1e-12)
    assert st == 0
    with LbmSolver(norm) as s:
        s.set_design(raw)
        s.forward()
        g_n, rep_n = s.gradient(w, mode="steady", tolerance=1e-10)
        g_k, rep_k = s.gradient(w, mode="steady", tolerance=1e-10, steady_solver="bicgstab")
    assert rep_n.converged and rep_k.converged
    assert rep_k.residual <= 1e-10
    assert rel_l2(g_k, g_n) < 1e-6, rel_l2(g_k, g_n)
    assert rel_l2(g_k, g_ref) < 1e-4, rel_l2(g_k, g_ref)


def test_bicgstab_needs_fp32_vectors(gpu_lib):
    norm = normalize(_problem("trt", "D3Q19", None, steps=50))
    with LbmSolver(norm) as s:
        s.set_design(workloads.uniform_design(norm.shape, 1))
        s.forward()
        with pytest.raises(ContractError, match="float32"):
            s.gradient(workloads.objective_weights(), mode="steady", lambda_storage="float16",
                       steady_solver="bicgstab")


def test_bicgstab_on_the_128_channel(gpu_lib):
    """The 128^3 channel workload (5000 forward steps): the same gradient as
    the Neumann series with at least three times fewer operator applications."""
    shape, steps, coll, _, _ = workloads.CONFIGS["channel128_trt"]
    norm = normalize(workloads.channel_problem(shape=shape, steps=steps, collision=coll))
    w = workloads.objective_weights()
    with LbmSolver(norm) as s:
        s.set_design(workloads.uniform_design(shape, 0))
        s.forward()
        g_n, rep_n = s.gradient(w, mode="steady", tolerance=1e-10, check_every=20)
        g_k, rep_k = s.gradient(w, mode="steady", tolerance=1e-10, steady_solver="bicgstab")
    print({"neumann": rep_n.iterations, "bicgstab": rep_k.iterations, "rel_l2": rel_l2(g_k, g_n),
           "neumann_ms": rep_n.adjoint_ms, "bicgstab_ms": rep_k.adjoint_ms})
    assert rep_n.converged and rep_k.converged
    assert rel_l2(g_k, g_n) < 1e-6, rel_l2(g_k, g_n)
    assert 3 * rep_k.iterations <= rep_n.iterations, (rep_k.iterations, rep_n.iterations)
