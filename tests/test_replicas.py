"""The replica path of bench.py on CPU: two gloo ranks, barrier and the
max-over-ranks of per-rank times."""
import os
import socket

import pytest
import torch.multiprocessing as mp


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    os.environ.update(RANK=str(rank), WORLD_SIZE=str(world), LOCAL_RANK=str(rank), MASTER_ADDR="127.0.0.1",
                      MASTER_PORT=str(port))
    from implexity_b200 import replicas

    r, w, _ = replicas.init("gloo", timeout_s=30)
    assert (r, w) == (rank, world)
    replicas.barrier()
    out[rank] = replicas.max_over_ranks(1.5 + rank)
    replicas.finalize()


@pytest.mark.parametrize("world", [2])
def test_max_over_ranks_gloo(world):
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
        assert p.exitcode == 0
    assert dict(out) == {r: 1.5 + world - 1 for r in range(world)}


def test_single_process_is_identity():
    from implexity_b200 import replicas

    assert replicas.max_over_ranks(3.25) == 3.25
