"""Batched AMR block lists on the GPU: one persistent launch per RK stage over
an uneven list of mixed-size blocks, against the CPU oracle evaluated block by
block (each block is an independent padded grid with its own spacing)."""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _small_pool(count=5, seed=7, ng=3):
    from bssn3d_b200 import amr
    from bssn3d_b200.initial_data import Puncture
    punct = [Puncture(0.909, (-0.5, 0.0, 0.0)), Puncture(0.0909, (5.0, 0.0, 0.0))]
    blocks = amr.nested_blocks(count, 3, punct, 16.0, 0.25, seed=seed, sizes=(8, 12, 16),
                               probs=(0.4, 0.3, 0.3), ng=ng)
    pool = amr.BlockPool(blocks)
    return pool, pool.initial_state(punct, seed=3), punct


def _S(h, dt, t=0.0):
    from bssn3d_b200.fused_rhs import pack_S
    return pack_S(2.0, 0.06, dt, h, 0.6, 20.0, t, (1, 1, 1, 1), (1, 0), h, h)


@pytest.mark.parametrize("variant", [0, 1, 2, 3])
def test_batched_rhs_vs_oracle(variant):
    from bssn3d_b200 import amr
    pool, U, _ = _small_pool()
    evo = amr.BatchedEvolution(pool, ko_sigma=0.1, ko_order=6, variant=variant)
    dt = 0.25 * min(b.h for b in pool.blocks)
    out = evo.rhs(torch.from_numpy(U).cuda(), evo.scalars(0.3, dt)).cpu().numpy()
    for i, b in enumerate(pool.blocks):
        ref = O.rhs(pool.gather(U, i), _S(b.h, dt, 0.3))
        assert O.normwise_rel(pool.gather(out, i), ref).max() < 1e-12, (variant, i)


def test_batched_rk4_step_vs_oracle_and_per_block():
    from bssn3d_b200 import amr
    pool, U, _ = _small_pool(count=6, seed=11)
    dt = 0.25 * min(b.h for b in pool.blocks)
    evo = amr.BatchedEvolution(pool, ko_sigma=0.1, ko_order=6, variant=0)
    Ud = torch.from_numpy(U).cuda()
    new = evo.evolve(Ud, dt, 1, t0=0.0).cpu().numpy()
    # one launch per block per stage with the uniform kernel gives the same bytes
    Up = Ud.clone()
    evo.per_block_step_inplace(Up, evo.block_scalars(0.0, dt))
    np.testing.assert_array_equal(Up.cpu().numpy(), new)
    for i, b in enumerate(pool.blocks):
        ref = O.rk4_step(pool.gather(U, i), _S(b.h, dt, 0.0), ko_sigma=0.1, ko_order=6)
        assert O.normwise_rel_grouped(pool.gather(new, i), ref).max() < 1e-12, i


def test_batched_variants_agree_and_repeat_bit_identically():
    from bssn3d_b200 import amr
    pool, U, _ = _small_pool(count=4, seed=5)
    dt = 0.25 * min(b.h for b in pool.blocks)
    Ud = torch.from_numpy(U).cuda()
    evo = amr.BatchedEvolution(pool, ko_sigma=0.1, ko_order=6, variant=0)
    base = evo.evolve(Ud, dt, 2).cpu().numpy()
    for _ in range(4):
        np.testing.assert_array_equal(evo.evolve(Ud, dt, 2).cpu().numpy(), base)
    for v in (1, 2, 3):
        evo.set_variant(v)
        other = evo.evolve(Ud, dt, 2).cpu().numpy()
        assert np.abs(other - base).max() <= 1e-13 * np.abs(base).max()


def test_batched_ko8_ghost4():
    from bssn3d_b200 import amr
    pool, U, _ = _small_pool(count=3, seed=2, ng=4)
    dt = 0.25 * min(b.h for b in pool.blocks)
    evo = amr.BatchedEvolution(pool, ko_sigma=0.1, ko_order=8, variant=2)
    new = evo.evolve(torch.from_numpy(U).cuda(), dt, 1).cpu().numpy()
    for i, b in enumerate(pool.blocks):
        ref = O.rk4_step(pool.gather(U, i), _S(b.h, dt), ko_sigma=0.1, ko_order=8, ng=4)
        assert O.normwise_rel_grouped(pool.gather(new, i), ref).max() < 1e-12


def test_autotune_picks_a_variant_and_block_order():
    from bssn3d_b200 import amr
    pool, U, _ = _small_pool(count=8, seed=1)
    evo = amr.BatchedEvolution(pool, ko_sigma=0.1, ko_order=6)
    times = amr.autotune(evo, torch.from_numpy(U).cuda(), 0.01, reps=2)
    assert sorted(times) == [(v, o) for v in range(4) for o in sorted(amr.BatchedEvolution.ORDERS)]
    assert (evo.variant, evo.order) == min(times, key=times.get)


@pytest.mark.parametrize("ghosts", ["evolve", "exchange"])
def test_block_order_and_one_launch_per_block_give_the_same_bytes(ghosts):
    """The block-to-CTA mapping and the launch structure change only which CTA
    computes a tile, never its arithmetic: every form gives the same bytes."""
    from bssn3d_b200 import amr
    pool, U, _ = _small_pool(count=6, seed=11)
    dt = 0.25 * min(b.h for b in pool.blocks)
    Ud = torch.from_numpy(U).cuda()
    evo = amr.BatchedEvolution(pool, ko_sigma=0.1, ko_order=6, variant=2, ghosts=ghosts)
    base = evo.evolve(Ud, dt, 2).cpu().numpy()
    evo.set_variant(2, "size")
    assert evo.launch_order("size") != evo.launch_order("pool")
    np.testing.assert_array_equal(evo.evolve(Ud, dt, 2).cpu().numpy(), base)
    g, U_g, _ = evo.capture_per_block(Ud, evo.scalars(0.0, dt))
    for _ in range(2):
        g.replay()
    np.testing.assert_array_equal(U_g.cpu().numpy(), base)
