"""Ghost exchange across ranks for a block list split over processes, on the
CPU: the per-rank layouts partition the global fill plan exactly, every
receive has its matching send, and gloo ranks that exchange their mirrors
level by level and run their own fill boxes reproduce the single-process
oracle fill bit for bit."""

import os
import socket

import numpy as np
import pytest
import torch

from oracle import amr_oracle as A


def _blocks(seed=7, count=14):
    from bssn3d_b200 import amr
    from bssn3d_b200.initial_data import Puncture
    punct = [Puncture(0.909, (-0.5, 0.0, 0.0)), Puncture(0.0909, (1.0, 0.0, 0.0))]
    return amr.nested_blocks(count, 3, punct, 4.0, 0.25, seed=seed, sizes=(6, 8, 10),
                             probs=(0.4, 0.4, 0.2), ng=3)


def _run_level(pool, lists, level, state):
    """Execute one level's boxes on a flat state with numpy (one launch)."""
    from bssn3d_b200 import ghosts as G
    geo = A.geometry_of(pool)
    by_off = {g.offset: g for g in geo}
    snap = state.copy()
    for lvl, ops in lists:
        if lvl != level:
            continue
        for op in ops:
            D, S = by_off[op.dst_off], by_off[op.src_off]
            lo, hi, sh = list(op.lo), list(op.hi), list(op.shift)
            d = np.indices([hi[k] - lo[k] for k in range(3)]).reshape(3, -1).T + lo
            src = S.view(snap)
            if op.kind == G.COPY:
                s = d + sh
                val = src[:, s[:, 0], s[:, 1], s[:, 2]]
            elif op.kind == G.RESTRICT:
                s = 2 * d + sh
                val = src[:, s[:, 0], s[:, 1], s[:, 2]]
            else:
                g = d + sh
                val = A.refine(src)[:, g[:, 0], g[:, 1], g[:, 2]]
            D.view(state)[:, d[:, 0], d[:, 1], d[:, 2]] = val


@pytest.mark.parametrize("world", [2, 3])
def test_rank_layouts_partition_the_plan(world):
    from bssn3d_b200 import amr, ghosts
    from bssn3d_b200.parallel import RankLayout
    blocks = _blocks()
    gplan = ghosts.GhostPlan(amr.BlockPool(blocks))
    total = sum(len(ops) for _, ops in gplan.fill_lists)
    lays = [RankLayout(blocks, world, r, plan=gplan) for r in range(world)]
    assert sum(len(ops) for L in lays for _, ops in L.fill_lists) == total
    owned = sorted(g for L in lays for g in (L.index[i] for i in L.owned))
    assert owned == list(range(len(blocks)))
    for q, L in enumerate(lays):
        for lvl, pairs in L.recv.items():
            for p, j in pairs:
                assert p != q and (q, j) in lays[p].send[lvl]
        for lvl, pairs in L.send.items():
            for q2, j in pairs:
                assert (q, j) in lays[q2].recv[lvl]
        mirrors = {j for pairs in L.recv.values() for _, j in pairs}
        assert set(L.index) == set(L.parts[q]) | mirrors
    assert any(L.recv[lvl] for L in lays for lvl in L.levels)   # the split does cut the fill


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, seed, out, packed=False):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from bssn3d_b200 import amr
        from bssn3d_b200.parallel import RankLayout
        blocks = _blocks()
        gpool = amr.BlockPool(blocks)
        state = np.random.default_rng(seed).standard_normal(gpool.size)
        lay = RankLayout(blocks, world, rank)
        local = torch.zeros(lay.pool.size, dtype=torch.float64)
        for i in lay.owned:                         # only its own blocks start filled
            g = lay.index[i]
            o = int(gpool.offsets[g])
            lay.block_view(local, g).copy_(torch.from_numpy(state[o:o + 24 * blocks[g].points]))
        arr = local.numpy()
        for lvl in lay.levels:
            if packed:
                lay.exchange_packed(local, lvl)
            else:
                lay.exchange(local, lvl)
            _run_level(lay.pool, lay.fill_lists, lvl, arr)
        want = A.fill(state, A.geometry_of(gpool))
        ok = True
        for i in lay.owned:
            g = lay.index[i]
            o = int(gpool.offsets[g])
            ok &= np.array_equal(lay.block_view(local, g).numpy(), want[o:o + 24 * blocks[g].points])
        out[rank] = int(ok)
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,packed", [(2, False), (3, False), (2, True), (3, True)])
def test_gloo_ranks_fill_like_one_process(world, packed):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, 3, out, packed)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    assert dict(out) == {r: 1 for r in range(world)}


@pytest.mark.parametrize("world", [2, 3])
def test_packed_exchange_moves_only_the_read_points(world):
    """The packed halos are a subset of the whole mirrored blocks, cover
    every point a rank's fill boxes read, and move fewer bytes."""
    from bssn3d_b200 import amr, ghosts
    from bssn3d_b200.parallel import RankLayout, read_box
    blocks = _blocks()
    gplan = ghosts.GhostPlan(amr.BlockPool(blocks))
    lays = [RankLayout(blocks, world, r, plan=gplan) for r in range(world)]
    packed = sum(L.exchange_bytes(True) for L in lays)
    whole = sum(L.exchange_bytes(False) for L in lays)
    assert 0 < packed < whole
    for L in lays:
        for lvl, ops in L.fill_lists:
            for op in ops:
                g = L.index[[int(o) for o in L.pool.offsets].index(op.src_off)]
                if g in L.parts[L.rank]:
                    continue
                pts = set(L._reads[L.rank][(lvl, g)].tolist())
                (x0, x1), (y0, y1), (z0, z1) = read_box(op)
                sy, sz = op.src_s[1], op.src_s[2]
                for x in (x0, x1 - 1):
                    for y in (y0, y1 - 1):
                        for z in (z0, z1 - 1):
                            assert (x * sy + y) * sz + z in pts


def _restrict_worker(rank, world, port, seed, out):
    """Restriction across ranks: each rank injects (packed exchange of the
    remote fine points, then its own restriction boxes) and its coarse
    blocks equal the single-process injection."""
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from bssn3d_b200 import amr, ghosts
        from bssn3d_b200.parallel import RankLayout
        blocks = _blocks()
        gpool = amr.BlockPool(blocks)
        gplan = ghosts.GhostPlan(gpool, restrict=True)
        state = np.random.default_rng(seed).standard_normal(gpool.size)
        want = state.copy()
        for lvl, _ in gplan.restrict_lists:          # the single process, finest first
            _run_level(gpool, gplan.restrict_lists, lvl, want)
        lay = RankLayout(blocks, world, rank, plan=gplan)
        local = torch.zeros(lay.pool.size, dtype=torch.float64)
        for i in lay.owned:
            g = lay.index[i]
            o = int(gpool.offsets[g])
            lay.block_view(local, g).copy_(torch.from_numpy(state[o:o + 24 * blocks[g].points]))
        arr = local.numpy()
        for lvl in lay.restrict_levels:
            lay.exchange_packed(local, lvl, phase="restrict")
            _run_level(lay.pool, lay.restrict_lists, lvl, arr)
        ok = True
        for i in lay.owned:
            g = lay.index[i]
            o = int(gpool.offsets[g])
            ok &= np.array_equal(lay.block_view(local, g).numpy(), want[o:o + 24 * blocks[g].points])
        out[rank] = (int(ok), lay.exchange_bytes(True, "restrict"), lay.exchange_bytes(False, "restrict"))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_ranks_restrict_like_one_process(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_restrict_worker, args=(r, world, port, 5, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    res = dict(out)
    assert all(res[r][0] == 1 for r in range(world))
    sent = sum(res[r][1] for r in range(world))
    assert 0 < sent < sum(res[r][2] for r in range(world))   # the split cuts the injection, packed < whole
