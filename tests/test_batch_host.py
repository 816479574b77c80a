"""Host logic of batched scans: seeded draws, cost-balanced partition across
ranks, and the end-of-run gather / max-over-ranks timing, the multi-rank
parts on 2 gloo ranks (CPU)."""
import socket

import numpy as np
import pytest

from lcode3d_b200 import batch as B


def test_scan_specs_seeded_and_in_range():
    a = B.scan_specs(32, 7)
    assert a == B.scan_specs(32, 7)
    assert a != B.scan_specs(32, 8)
    for s in a:
        N = s['grid_steps']
        assert N in B.GRIDS
        assert s['grid_step_size'] == 16.0 / (N - 1)
        assert 0.01 <= s['amplitude'] <= 1.0
        assert 0.5 <= s['sigma_r'] <= 2.0
        assert 0.5 <= s['length_factor'] <= 1.5
    assert len({s['grid_steps'] for s in a}) > 1


@pytest.mark.parametrize('world', [1, 2, 3, 4, 8])
def test_partition_covers_and_balances(world):
    specs = B.scan_specs(32, 1)
    parts = B.partition(specs, world)
    assert len(parts) == world
    assert sorted(i for p in parts for i in p) == list(range(32))
    loads = [sum(B.cost(specs[i]) for i in p) for p in parts]
    assert max(loads) - min(loads) <= max(B.cost(s) for s in specs)
    assert parts == B.partition(specs, world)   # deterministic


def test_single_rank_helpers():
    assert B.max_over_ranks(3.5) == 3.5
    h = {0: np.arange(3.0)}
    assert B.gather_histories(h) == h


def _free_port():
    with socket.socket() as s:
        s.bind(('127.0.0.1', 0))
        return s.getsockname()[1]


def _worker(rank, world, port, q):
    import torch.distributed as dist
    dist.init_process_group('gloo', rank=rank, world_size=world,
                            init_method=f'tcp://127.0.0.1:{port}')
    try:
        specs = B.scan_specs(12, 3)
        mine = B.partition(specs, world)[rank]
        # stand-in for the Ez(0,0) histories a rank's simulations produce
        local = {i: np.full(5, float(i)) for i in mine}
        merged = B.gather_histories(local, dist)
        slowest = B.max_over_ranks(float(rank + 1), dist)
        q.put((rank, mine, sorted(merged), [float(merged[k][0]) for k in sorted(merged)], slowest))
    finally:
        dist.destroy_process_group()


def test_two_rank_partition_gather_and_timing():
    import torch.multiprocessing as mp
    ctx = mp.get_context('spawn')
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    results = [q.get(timeout=180) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    mine = {}
    for rank, part, keys, firsts, slowest in results:
        mine[rank] = part
        assert keys == list(range(12))                  # every rank sees every history
        assert firsts == [float(k) for k in range(12)]
        assert slowest == 2.0                           # max over ranks of (rank + 1)
    assert sorted(mine[0] + mine[1]) == list(range(12))
    assert not set(mine[0]) & set(mine[1])
