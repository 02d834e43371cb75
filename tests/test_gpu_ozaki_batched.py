"""Ozaki INT8 derivatives over a block list (bssn_b200_batch_ozaki_derivatives)
and the RK4 stage from precomputed derivatives (bssn_b200_batch_rk4_stage_derivs):
with whole blocks covered the batched bundle equals the single-grid Ozaki
bundle block by block, bit for bit; with ghost exchange the covered
interiors agree with the float64 derivatives within the digit-split bound;
RK4 steps through the Ozaki path track the float64 block-list path."""

import numpy as np
import pytest
import torch

from oracle import amr_oracle as A
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pool(ng=3, count=10, seed=7):
    from bssn3d_b200 import amr
    from bssn3d_b200.initial_data import Puncture
    punct = [Puncture(0.909, (-0.5, 0.0, 0.0)), Puncture(0.0909, (1.0, 0.0, 0.0))]
    blocks = amr.nested_blocks(count, 3, punct, 6.0, 0.25, seed=seed, sizes=(8, 10, 12),
                               probs=(0.4, 0.4, 0.2), ng=ng)
    return amr.BlockPool(blocks), punct


def _S(h, dt=0.01, t=0.0):
    from bssn3d_b200.fused_rhs import device_scalars, pack_S
    return device_scalars(pack_S(2.0, 0.06, dt, h, 0.6, 20.0, t, (1, 1, 1, 1), (1, 0), h, h),
                          torch.device("cuda"))


def _block(pool, X, i):
    b = pool.blocks[i]
    o = int(pool.offsets[i])
    return X[o:o + 24 * b.points].view((24,) + tuple(b.shape))


@pytest.mark.parametrize("ko_order", [6, 8])
def test_whole_blocks_equal_single_grid_bundle(ko_order):
    from bssn3d_b200.ozaki import BatchedOzakiEvolution, OzakiDerivatives
    pool, punct = _pool(ng=4)
    U = torch.from_numpy(pool.initial_state(punct, seed=1)).cuda()
    evo = BatchedOzakiEvolution(pool, k=6, ko_sigma=0.1, ko_order=ko_order, ghosts="evolve")
    evo.derivatives(U, evo.scalars(0.0, 0.01))
    torch.cuda.synchronize()
    evo.check()
    for i, blk in enumerate(pool.blocks):
        oz = OzakiDerivatives(blk.shape, 6)
        ref = oz.derivatives(_block(pool, U, i), _S(blk.h), ko_sigma=0.1, ko_order=ko_order)
        assert torch.equal(evo.derivative_view(i), ref), i


def test_covered_interiors_equal_cpu_restatement():
    """With ghost exchange every block's interior slots equal the numpy
    restatement of the passes over that block's covered boxes, bit for bit."""
    from bssn3d_b200.ozaki import BatchedOzakiEvolution
    from oracle import ozaki_oracle as Z
    pool, punct = _pool(count=6)
    Y = torch.from_numpy(pool.initial_state(punct, seed=1)).cuda()
    evo = BatchedOzakiEvolution(pool, k=6, ko_sigma=0.1, ko_order=6, ghosts="exchange")
    evo.fill(Y)
    evo.derivatives(Y, evo.scalars(0.0, 0.01))
    torch.cuda.synchronize()
    evo.check()
    for i, blk in enumerate(pool.blocks):
        g = blk.ng
        want = Z.bundle(_block(pool, Y, i).cpu().numpy(), blk.h, 6, ko_sigma=0.1, ko_order=6, core=g)
        got = evo.derivative_view(i).cpu().numpy()
        I = (slice(None),) + (slice(g, -g),) * 3
        assert np.array_equal(got[I], want[I]), i


def test_covered_interiors_match_fp64_derivatives():
    from bssn3d_b200.fused_rhs import derivatives
    from bssn3d_b200.ozaki import BatchedOzakiEvolution
    pool, punct = _pool()
    U = torch.from_numpy(pool.initial_state(punct, seed=1)).cuda()
    Y = U.clone()
    errs = {}
    for k in (5, 8):
        evo = BatchedOzakiEvolution(pool, k=k, ko_sigma=0.1, ko_order=6, ghosts="exchange")
        evo.fill(Y)
        evo.derivatives(Y, evo.scalars(0.0, 0.01))
        torch.cuda.synchronize()
        evo.check()
        worst = 0.0
        for i, blk in enumerate(pool.blocks):
            g = blk.ng
            F = _block(pool, Y, i)
            ref = derivatives(F.contiguous(), _S(blk.h), ko_sigma=0.1, ko_order=6)
            got = evo.derivative_view(i)
            I = (slice(g, -g),) * 3
            fmax = F.abs().amax(dim=(1, 2, 3)).cpu().numpy()
            for s in range(162):
                f = s // 3 if s < 72 else (None if s < 138 else s - 138)
                order = 1 if (s < 72 or s >= 138) else 2
                scale = (fmax.max() if f is None else fmax[f]) / blk.h ** order
                if scale == 0:
                    continue
                e = float((got[s][I] - ref[s][I]).abs().max()) / scale
                worst = max(worst, e)
        errs[k] = worst
    # split residual 2^(e-7k-1) per value: k = 8 sits at float64 rounding, k = 5 well above it
    assert errs[8] < 1e-13
    assert errs[5] > errs[8]


@pytest.mark.parametrize("ko_order", [6, 8])
def test_rk4_steps_track_the_fp64_block_path(ko_order):
    from bssn3d_b200 import amr
    from bssn3d_b200.ozaki import BatchedOzakiEvolution
    ng = max(3, ko_order // 2)
    pool, punct = _pool(ng=ng)
    U = torch.from_numpy(pool.initial_state(punct, seed=2)).cuda()
    dt = 0.25 * min(b.h for b in pool.blocks)
    ref = amr.BatchedEvolution(pool, ko_sigma=0.1, ko_order=ko_order, ghosts="exchange").evolve(U, dt, 2)
    oz = BatchedOzakiEvolution(pool, k=8, ko_sigma=0.1, ko_order=ko_order, ghosts="exchange")
    got = oz.evolve(U, dt, 2)
    torch.cuda.synchronize()
    oz.check()
    assert bool(torch.isfinite(got).all())
    gn, rn = got.cpu().numpy(), ref.cpu().numpy()
    for i, G in enumerate(A.geometry_of(pool)):
        I = (slice(None),) + (slice(G.ng, -G.ng),) * 3
        assert O.normwise_rel_grouped(G.view(gn)[I], G.view(rn)[I]).max() < 1e-10, i


def test_graph_replay_equals_eager_steps():
    from bssn3d_b200.ozaki import BatchedOzakiEvolution
    pool, punct = _pool()
    U = torch.from_numpy(pool.initial_state(punct, seed=3)).cuda()
    dt = 0.25 * min(b.h for b in pool.blocks)
    oz = BatchedOzakiEvolution(pool, k=6, ko_sigma=0.1, ko_order=6, ghosts="exchange")
    S = oz.scalars(0.0, dt)
    eager = U.clone()
    oz.seed_buffers(eager)
    for _ in range(2):
        oz.step_inplace(eager, S)
        oz.advance_time(S)
    got = oz.evolve(U, dt, 2)
    torch.cuda.synchronize()
    oz.check()
    assert torch.equal(got, eager)


def test_choose_k_takes_the_smallest_k_within_the_bar():
    """The autotuner's digit-count knob: errors of the block-list RHS fall
    with k, and the chosen k is the first whose worst field meets the bar."""
    from bssn3d_b200.ozaki import choose_k
    pool, punct = _pool(count=6, seed=3)
    U = torch.from_numpy(pool.initial_state(punct, seed=2)).cuda()
    dt = 0.25 * min(b.h for b in pool.blocks)
    k, errs = choose_k(pool, U, dt, ks=(4, 5, 6, 7, 8), bar=1e-10)
    assert errs[4] > errs[5] > errs[6] > errs[7] > errs[8]
    assert k == min(q for q in errs if errs[q] <= 1e-10)
    assert errs[8] < 1e-12
