"""Slab split of one uniform block across ranks, on the CPU: the plane
ranges partition the array and balance the evaluated planes; gloo ranks
that each step their slab (the oracle's RHS + KO as the stage rate) and
exchange halo planes after every stage reproduce the single-process RK4
steps bit for bit on their owned planes, and the gathered state equals the
single-process state."""

import os
import socket

import numpy as np
import pytest
import torch

from oracle import oracle as O


def test_slab_ranges_partition_and_balance():
    from bssn3d_b200.slabs import SlabLayout, slab_ranges
    for Sx, world, halo in [(134, 2, 3), (134, 3, 3), (134, 8, 3), (70, 4, 4), (16, 3, 3), (20, 1, 3)]:
        rng = slab_ranges(Sx, world, halo)
        assert rng[0][0] == 0 and rng[-1][1] == Sx
        assert all(rng[i][1] == rng[i + 1][0] for i in range(world - 1))
        lays = [SlabLayout(Sx, world, r, halo) for r in range(world)]
        evaluated = [L.local_planes for L in lays]
        assert max(evaluated) - min(evaluated) <= 1
        for L in lays:
            assert L.b - L.a >= (halo if world > 1 else 1)
            for q, planes in L.sends:           # every send is a matching receive
                assert (L.rank, planes) in lays[q].recvs
            if world > 1:
                assert L.exchange_bytes(5, 7) == 8 * 24 * halo * 35 * len(L.sends)
    with pytest.raises(ValueError):
        slab_ranges(12, 4, 3)                  # slabs thinner than the halo


def cpu_stage(stage, U, Y, ACC, YNEXT, S):
    """One RK4 stage on the CPU with the oracle's rate (RHS + KO6, sigma 0.1):
    the stage kernel's recurrence (k1..k4 folded into ACC, enforcement after
    the last stage)."""
    s = S.numpy().copy()
    dt = s[2]
    s[6] = s[6] + (0.0, 0.5, 0.5, 1.0)[stage] * dt
    k = torch.from_numpy(O.rate(Y.numpy(), s, ko_sigma=0.1, ko_order=6))
    if stage == 0:
        ACC.copy_(k)
        YNEXT.copy_(U + 0.5 * dt * k)
    elif stage in (1, 2):
        ACC.add_(2.0 * k)
        YNEXT.copy_(U + (0.5 if stage == 1 else 1.0) * dt * k)
    else:
        YNEXT.copy_(torch.from_numpy(O.enforce((U + dt / 6.0 * (ACC + k)).numpy())))


def _state():
    from bssn3d_b200 import initial_data as ID
    return ID.workload(0, n=10)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, nsteps, out):
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from bssn3d_b200.slabs import SlabEvolution
        grid, U, dt = _state()
        U = torch.from_numpy(U)
        one = SlabEvolution(grid, world=1, rank=0, stage_fn=cpu_stage)
        want = one.evolve(U, dt, nsteps)
        evo = SlabEvolution(grid, world=world, rank=rank, stage_fn=cpu_stage)
        got = evo.evolve(evo.local(U), dt, nsteps)
        lay = evo.layout
        own_ok = torch.equal(evo.owned(got), want[:, lay.a:lay.b])
        halo_ok = torch.equal(got, want[:, lay.local_slice()])   # halos current after the last exchange
        full_ok = torch.equal(evo.gather(got), want)
        out[rank] = (int(own_ok), int(halo_ok), int(full_ok), lay.exchange_bytes(*U.shape[2:]))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_gloo_slab_ranks_step_like_one_process(world):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    out = ctx.Manager().dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, 2, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
        assert p.exitcode == 0
    res = dict(out)
    assert [res[r][:3] for r in range(world)] == [(1, 1, 1)] * world
    assert all(res[r][3] > 0 for r in range(world))


def test_local_exchange_matches_owner_planes():
    """The one-process exchange copies exactly the neighbours' owned planes."""
    from bssn3d_b200.slabs import SlabLayout, exchange_halos_local
    Sx, world, halo = 23, 3, 3
    G = torch.arange(24 * Sx * 2 * 3, dtype=torch.float64).reshape(24, Sx, 2, 3)
    lays = [SlabLayout(Sx, world, r, halo) for r in range(world)]
    Ys = [torch.full((24, L.local_planes, 2, 3), -1.0, dtype=torch.float64) for L in lays]
    for L, Y in zip(lays, Ys):
        Y[:, L.owned_slice()] = G[:, L.a:L.b]
    exchange_halos_local(lays, Ys)
    for L, Y in zip(lays, Ys):
        assert torch.equal(Y, G[:, L.local_slice()])
