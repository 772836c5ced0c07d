"""CPU (gloo, world_size 2) test of the multi-rank host logic of bench.py:
each rank builds its own replica (replicas only, no data-path collective),
and the step time is the maximum over ranks, reduced with one all_reduce."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, out):
    import importlib.util
    import sys
    sys.path.insert(0, ROOT)
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    spec = importlib.util.spec_from_file_location("bench", os.path.join(ROOT, "bench.py"))
    bench = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(bench)
    pos, q, box = bench.make_workload(seed=rank, box=16.0)
    t_ms = 1.0 + rank  # stand-in for the rank's measured step time
    tt = torch.tensor([t_ms])
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    out[rank] = (float(q.sum()), len(q), float(pos[:5].sum()), float(tt.item()))
    dist.destroy_process_group()


@pytest.mark.timeout(120)
def test_two_rank_replicas_and_max_time():
    world = 2
    port = _free_port()
    with mp.Manager() as m:
        out = m.dict()
        mp.spawn(_worker, args=(world, port, out), nprocs=world, join=True)
        res = dict(out)
    assert len(res) == 2
    for rank in range(world):
        qsum, n, _, tmax = res[rank]
        assert qsum == 0.0 and n == int(0.5 * 16 ** 3)
        assert tmax == 2.0  # max over ranks
    assert res[0][2] != res[1][2]  # rank-seeded, independent replicas
