"""Ensemble sharding over ranks (host logic, no GPU): whole instances placed
by the longest-processing-time greedy rule on their cell counts, per-instance
results gathered to rank 0, max over ranks -- with two gloo ranks on CPU."""
import os
import socket

import numpy as np
import pytest


def test_assignment_properties():
    import pic_configs as C
    import sharding as S
    ws = C.cfg5_instances()
    cells = [w.nx * w.ny for w in ws]
    assert S.assign(cells, 1) == [0] * len(cells)
    for world in (2, 3, 4, 8):
        r = S.assign(cells, world)
        assert r == S.assign(cells, world)                  # every rank computes the same
        assert sorted(sum((S.local(cells, world, k) for k in range(world)), [])) == list(range(64))
        ld = S.loads(cells, world)
        assert max(ld) - min(ld) <= max(cells)
        # LPT is within 4/3 of the best possible makespan
        assert max(ld) <= (4 / 3) * max(sum(cells) / world, max(cells)) + 1e-9
    # more ranks than instances: the extra ranks hold none
    r = S.assign([5.0, 3.0], 4)
    assert sorted(r) == [0, 1] and S.local([5.0, 3.0], 4, 3) == []
    with pytest.raises(ValueError):
        S.assign([1.0], 0)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _worker(rank, world, port, q):
    import datetime
    import sys
    here = os.path.dirname(os.path.abspath(__file__))
    sys.path[:0] = [os.path.join(os.path.dirname(here), "bmp-6th-sem_b200")]
    import torch.distributed as dist
    import sharding as S
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=60))
    try:
        cells = [float(c) for c in np.random.default_rng(3).integers(100, 1000, 17)]
        mine = S.local(cells, world, rank)
        metrics = {i: {"cells": cells[i], "rank": rank} for i in mine}
        got = S.gather_metrics(metrics)
        mx = S.max_over_ranks(sum(cells[i] for i in mine))
        tot = S.sum_over_ranks(len(mine))
        if rank == 0:
            q.put((sorted(got), {i: v["rank"] for i, v in got.items()}, mx, tot,
                   S.assign(cells, world), max(S.loads(cells, world))))
        else:
            assert got is None
    finally:
        dist.destroy_process_group()


def test_two_gloo_ranks_gather_every_instance():
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    keys, ranks, mx, tot, assign, max_load = q.get(timeout=10)
    assert keys == list(range(17))
    assert [ranks[i] for i in range(17)] == assign
    assert mx == max_load and tot == 17
