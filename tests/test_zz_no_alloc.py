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


CASES = [
    # a small channel with a solid block: 10 blocks, one cell per thread
    ("D3Q19", (20, 12, 10), 80),
    # 294 912 cells: the grid is capped at the 1024 blocks the static array
    # holds partials for, each thread covers several cells, and the last block
    # merges a full partials array
    ("D3Q19", (72, 64, 64), 10),
    ("D3Q27", (20, 12, 10), 80),
]


@pytest.mark.parametrize("lattice,shape,steps", CASES)
def test_noalloc_stats_match_forward_record(gpu_lib, lattice, shape, steps):
    import torch

    solid = np.zeros(shape, bool)
    solid[9:11, 5:7, 4:6] = True
    prob = workloads.channel_problem(shape=shape, steps=steps, collision="trt", lattice=lattice, solid=solid)
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
    # the same sums in FP64 on the host
    fluid = ~solid.ravel()
    assert abs(mass - f[fluid].sum()) <= 1e-6 * mass

    # a non-finite population in a solid cell is reported too, and the next
    # call on a clean state clears the flag again
    x = int(np.flatnonzero(solid.ravel())[0])
    f_bad = f_dev.clone()
    f_bad[3, x] = float("nan")
    for state, flag in ((f_bad, 1.0), (f_dev, 0.0)):
        st = gpu_lib.lbm_state_stats_noalloc(q, cells, _ptr(state), _ptr(solid_dev), _ptr(alpha_dev), acc, _ptr(out),
                                             stream)
        assert st == _abi.LBM_OK, gpu_lib.lbm_last_error(None).decode()
        torch.cuda.synchronize(dev)
        assert out.cpu().numpy()[3] == flag


def test_noalloc_rejects_oversized_state(gpu_lib):
    out = C.c_void_p(1)  # never dereferenced: the size check comes first
    st = gpu_lib.lbm_state_stats_noalloc(19, 1 << 27, C.c_void_p(1), None, None, None, out, None)
    assert st == _abi.LBM_E_CONTRACT
    assert "2^31" in gpu_lib.lbm_last_error(None).decode()
