"""Multi-GPU host logic on CPU: cell ranges and the step's one exchange
(min over ranks of the new chemistry time step), with world_size 2 over gloo.
Each rank integrates its range with the CPU oracle standing in for its GPU."""
import os
import socket

import numpy as np
import pytest

from gpufoam_b200 import mechanism as M
from gpufoam_b200 import sharding as S


def test_unweighted_ranges_partition():
    for n, world in [(0, 3), (7, 2), (100, 8), (5, 8)]:
        r = S.shard_ranges(n, world)
        assert r[0][0] == 0 and r[-1][1] == n
        assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
        sizes = [b - a for a, b in r]
        assert max(sizes) - min(sizes) <= 1


def test_weighted_ranges_balance():
    rng = np.random.default_rng(0)
    w = rng.integers(5, 200, size=1000).astype(float)  # attempts per cell
    r = S.shard_ranges(1000, 4, w)
    assert r[0][0] == 0 and r[-1][1] == 1000 and all(a[1] == b[0] for a, b in zip(r, r[1:]))
    loads = [w[a:b].sum() for a, b in r]
    assert max(loads) - min(loads) <= 2 * w.max()
    with pytest.raises(ValueError):
        S.shard_ranges(3, 2, [1.0, -1.0, 2.0])


def _worker(rank, world, port, n, out):
    import torch.distributed as dist

    from oracle.oracle import Oracle, ode_inputs
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    raw = M.h2_size(0)
    cells = M.make_cells(raw, n, seed=9)
    a, b = S.local_range(n, rank, world)
    _, dtc, _, _ = Oracle(raw, "port").cells(ode_inputs(34), cells[a:b], 1e-5, 1e-7)
    g = S.global_min_delta_t(float(dtc.min()) if b > a else float("inf"))
    out.put((rank, a, b, g))
    dist.barrier()
    dist.destroy_process_group()


def test_two_ranks_min_exchange():
    import multiprocessing as mp

    from oracle.oracle import Oracle, ode_inputs
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    n = 48
    procs = [ctx.Process(target=_worker, args=(r, 2, port, n, q)) for r in range(2)]
    for p in procs:
        p.start()
    res = sorted(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    raw = M.h2_size(0)
    _, dtc, _, _ = Oracle(raw, "port").cells(ode_inputs(34), M.make_cells(raw, n, seed=9), 1e-5, 1e-7)
    assert [(a, b) for _, a, b, _ in res] == S.shard_ranges(n, 2)
    assert res[0][3] == res[1][3] == float(dtc.min())
