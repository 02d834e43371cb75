"""Host-side logic of the batched AMR path (no GPU): block generation, pool
layout, the C-ABI planner (a pure host function), and the multi-rank block
partition exercised with gloo ranks on CPU."""

import os
import ctypes

import numpy as np
import pytest


def test_nested_blocks_seeded_and_mixed():
    from bssn3d_b200 import amr
    blocks, punct, dt = amr.workload(3)
    assert len(blocks) == 600
    sizes = sorted({b.n for b in blocks})
    assert sizes == [16, 24, 32]
    assert sorted({b.level for b in blocks}) == [0, 1, 2]
    assert dt == 0.25 * min(b.h for b in blocks)
    again, _, _ = amr.workload(3)
    assert [(b.n, b.origin, b.level) for b in again] == [(b.n, b.origin, b.level) for b in blocks]
    frac = np.mean([b.n == 16 for b in blocks])
    assert 0.4 < frac < 0.6


def test_pool_layout_and_plan_agree_with_c_planner():
    from bssn3d_b200 import amr, _lib
    blocks, _, _ = amr.workload(3, count=40)
    pool = amr.BlockPool(blocks)
    assert pool.offsets[0] == 0
    assert pool.size == sum(24 * b.points for b in blocks)
    shapes = {0: (4, 4, 16), 1: (2, 8, 16), 2: (4, 8, 8), 3: (8, 4, 8)}
    lib = _lib.load()
    for v, tile in shapes.items():
        ref_table, ref_tiles = pool.descriptors(tile)
        table, _ = pool.descriptors(tile)
        for b in table:
            b.tile0 = -1
        n = lib.bssn_b200_batch_plan(ctypes.addressof(table), len(blocks), v)
        assert n == ref_tiles
        assert [t.tile0 for t in table] == [t.tile0 for t in ref_table]


def test_planner_rejects_bad_tables():
    from bssn3d_b200 import amr, _lib
    blocks, _, _ = amr.workload(3, count=3)
    pool = amr.BlockPool(blocks)
    table, _ = pool.descriptors((4, 4, 16))
    table[1].h[0] = 0.0
    lib = _lib.load()
    assert lib.bssn_b200_batch_plan(ctypes.addressof(table), 3, 0) == -1
    assert "spacing" in lib.bssn_b200_last_error().decode()
    assert lib.bssn_b200_batch_plan(ctypes.addressof(table), 3, 9) == -1


def test_block_initial_data_is_brill_lindquist():
    from bssn3d_b200 import amr
    blocks, punct, _ = amr.workload(3, count=3)
    pool = amr.BlockPool(blocks)
    U = pool.initial_state(punct, seed=0)
    for i, b in enumerate(blocks):
        u = pool.gather(U, i)
        X, Y, Z = b.grid().mesh()
        psi = 1.0 + sum(p.mass / (2 * np.maximum(np.sqrt((X - p.position[0]) ** 2 + (Y - p.position[1]) ** 2
                                                         + (Z - p.position[2]) ** 2), 0.5 * b.h))
                        for p in punct)
        np.testing.assert_allclose(u[1], psi ** -4, rtol=1e-14)


def test_partition_balances_cost():
    from bssn3d_b200 import amr, parallel
    blocks, _, _ = amr.workload(4, count=300)
    parts = parallel.partition(blocks, 4)
    assert sorted(i for p in parts for i in p) == list(range(300))
    costs = [sum(blocks[i].points for i in p) for p in parts]
    assert max(costs) <= 1.1 * sum(costs) / 4 + max(b.points for b in blocks)


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    import torch
    from bssn3d_b200 import amr, parallel
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    blocks, _, _ = amr.workload(3, count=50)
    mine = parallel.local_blocks(blocks, rank, world)
    pts = torch.tensor([sum(b.interior_points for b in mine)], dtype=torch.float64)
    dist.all_reduce(pts)
    q.put((rank, len(mine), float(pts.item())))
    dist.destroy_process_group()


def test_gloo_ranks_cover_every_block_once():
    import multiprocessing as mp
    import socket
    from bssn3d_b200 import amr
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = [q.get(timeout=120) for _ in procs]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    blocks, _, _ = amr.workload(3, count=50)
    total = sum(b.interior_points for b in blocks)
    assert sum(n for _, n, _ in out) == 50
    assert all(t == total for _, _, t in out)
