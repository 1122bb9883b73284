"""lbm_state_stats_noalloc: admission statistics of a device-held state for
callers that cannot allocate device memory (code inside another framework's
memory pool, hosts with a fixed device budget).  The entry point keeps its scratch in a static device array,
so these callers pass only their own input and output buffers.

Checked against the existing entry points: the per-state admission record of
lbm_forward (lbm_trajectory) for the final state that lbm_get_populations
returns, within the 1e-5 relative tolerance of the parity tests, on two
calls in a row (the scratch keeps the previous call's contents; the second
call must not see them).  This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

from implexity_b200 import LbmSolver, _abi, normalize, workloads

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_noalloc_stats_match_forward_record(gpu_lib):
    import torch

    shape = (20, 12, 10)
    solid = np.zeros(shape, bool)
    solid[9:11, 5:7, 4:6] = True
    prob = workloads.channel_problem(shape=shape, steps=80, collision="trt", solid=solid)
    norm = normalize(prob)
    raw = workloads.uniform_design(shape, 5)
    with LbmSolver(norm) as s:
        s.set_design(raw)
        s.forward()
        f = s.populations()
        traj = s.trajectory()
        _, alpha = s.design()
        acc = (C.c_double * 3)(*s.acceleration_lattice)
        cells, q = s.cells, s.q

    dev = torch.device("cuda", 0)
    f_dev = torch.tensor(np.ascontiguousarray(f.T), dtype=torch.float32, device=dev)  # [q][cells]
    solid_dev = torch.tensor(solid.ravel().astype(np.uint8), device=dev)
    alpha_dev = torch.tensor(alpha.ravel(), dtype=torch.float32, device=dev)
    out = torch.empty(4, dtype=torch.float64, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    results = []
    for _ in range(2):
        out.fill_(np.nan)
        st = gpu_lib.lbm_state_stats_noalloc(q, cells, _ptr(f_dev), _ptr(solid_dev), _ptr(alpha_dev), acc, _ptr(out),
                                             stream)
        assert st == _abi.LBM_OK, gpu_lib.lbm_last_error(None).decode()
        torch.cuda.synchronize(dev)
        results.append(out.cpu().numpy().copy())
    np.testing.assert_array_equal(results[0], results[1])
    mass, min_pop, max_speed, nonfinite = results[0]
    assert nonfinite == 0.0
    assert abs(mass - traj["mass"][-1]) <= 1e-5 * traj["mass"][-1]
    assert abs(min_pop - traj["min_population"][-1]) <= 1e-5 * abs(traj["min_population"][-1])
    assert abs(max_speed - traj["max_speed"][-1]) <= 1e-5 * traj["max_speed"][-1]


def test_noalloc_rejects_oversized_state(gpu_lib):
    out = C.c_void_p(1)  # never dereferenced: the size check comes first
    st = gpu_lib.lbm_state_stats_noalloc(19, 1 << 27, C.c_void_p(1), None, None, None, out, None)
    assert st == _abi.LBM_E_CONTRACT
    assert "2^31" in gpu_lib.lbm_last_error(None).decode()
