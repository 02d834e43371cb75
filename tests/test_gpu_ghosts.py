"""AMR ghost exchange on the GPU (bssn_b200_fill and the batched exchange
step) against the CPU oracle of oracle/amr_oracle.py: the fill and the
restriction bit for bit, the reference's octree cross-level fill
(3D/tests/multipatch_amr/test_sync.py:42-65), polynomial exactness through
the kernel, and RK4 steps with ghosts refilled before every stage."""

import ctypes

import numpy as np
import pytest
import torch

from oracle import amr_oracle as A
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _pool(count=14, seed=11, domain=4.0, ng=3, sizes=(6, 8, 10), probs=(0.4, 0.4, 0.2)):
    from bssn3d_b200 import amr
    from bssn3d_b200.initial_data import Puncture
    punct = [Puncture(0.909, (-0.5, 0.0, 0.0)), Puncture(0.0909, (1.0, 0.0, 0.0))]
    blocks = amr.nested_blocks(count, 3, punct, domain, 0.25, seed=seed, sizes=sizes, probs=probs, ng=ng)
    return amr.BlockPool(blocks), punct


def _octree(corner, BS=16, NG=4):
    from bssn3d_b200 import amr
    parent = amr.Block(level=0, n=BS, origin=(0.0, 0.0, 0.0), h=1.0, ng=NG)
    child = amr.Block(level=1, n=BS, origin=tuple(c * BS / 2 for c in corner), h=0.5, ng=NG)
    return amr.BlockPool([parent, child])


def _gpu(pool, state, which="fill", restrict=False):
    from bssn3d_b200 import ghosts as G
    plan = G.GhostPlan(pool, restrict=restrict)
    dp = G.DevicePlan(plan, torch.device("cuda"))
    X = torch.from_numpy(state).cuda()
    dp.run(which, X, torch.cuda.current_stream().cuda_stream)
    return X.cpu().numpy()


@pytest.mark.parametrize("seed", [7, 11])
def test_fill_matches_oracle_bit_for_bit(seed):
    pool, _ = _pool(seed=seed)
    state = np.random.default_rng(seed).standard_normal(pool.size)
    geo = A.geometry_of(pool)
    assert np.array_equal(_gpu(pool, state), A.fill(state, geo))


def test_restriction_matches_oracle_bit_for_bit():
    pool, _ = _pool(seed=11)
    state = np.random.default_rng(4).standard_normal(pool.size)
    assert np.array_equal(_gpu(pool, state, "restrict", restrict=True), A.restrict(state, A.geometry_of(pool)))


def test_workload_fill_matches_oracle():
    from bssn3d_b200 import amr
    blocks, punct, _ = amr.workload(3, count=60)
    pool = amr.BlockPool(blocks)
    state = pool.initial_state(punct, seed=1)
    state += 1e-3 * np.random.default_rng(9).standard_normal(pool.size)
    assert np.array_equal(_gpu(pool, state), A.fill(state, A.geometry_of(pool)))


@pytest.mark.parametrize("corner", [(1, 0, 1), (0, 0, 0), (1, 1, 1)])
def test_octree_child_halo_is_prolongated_parent(corner):
    BS, NG = 16, 4
    pool = _octree(corner, BS, NG)
    geo = A.geometry_of(pool)
    state = np.random.default_rng(2).standard_normal(pool.size)
    geo[1].view(state)[:] = -7.0
    out = _gpu(pool, state)
    s = [NG + c * BS for c in corner]
    W = BS + 2 * NG
    want = A.refine(geo[0].view(state))[:, s[0]:s[0] + W, s[1]:s[1] + W, s[2]:s[2] + W]
    child = geo[1].view(out)
    halo = np.ones((W, W, W), bool)
    halo[NG:NG + BS, NG:NG + BS, NG:NG + BS] = False
    assert np.all(child[:, ~halo] == -7.0)                 # interior untouched
    assert np.array_equal(child[:, halo], want[:, halo])   # halo = refined parent, exactly
    assert np.array_equal(geo[0].view(out), geo[0].view(state))


def test_kernel_prolongation_reproduces_degree_five_polynomials():
    BS, NG, h = 16, 4, 0.37
    pool = _octree((0, 0, 0), BS, NG)
    geo = A.geometry_of(pool)
    W = BS + 2 * NG
    c = [np.array([0.4, -1.1, 0.7, 0.2, -0.3, 0.15]), np.array([-0.5, 0.9, -0.2, 0.6, 0.1, -0.25]),
         np.array([0.8, 0.3, -0.6, -0.1, 0.45, 0.05])]
    P = lambda k, x: sum(c[k][d] * x ** d for d in range(6))
    xp = (np.arange(W) - NG) * h
    state = np.zeros(pool.size)
    geo[0].view(state)[:] = np.einsum("i,j,k->ijk", P(0, xp), P(1, xp), P(2, xp))[None]
    child = geo[1].view(_gpu(pool, state))
    xf = (np.arange(W) - NG) * h / 2
    want = np.einsum("i,j,k->ijk", P(0, xf), P(1, xf), P(2, xf))
    # the low-x halo slab, away from the block edges in y and z (the
    # reference's deep-interior window, test_transfer.py:60-66)
    sl = (slice(0, NG),) + (slice(NG + 3, NG + BS - 3),) * 2
    assert np.max(np.abs(child[0][sl] - want[sl])) < 1e-9


def test_npoints_past_the_plan_writes_nothing_more():
    from bssn3d_b200 import _lib, ghosts as G
    pool, _ = _pool(seed=7)
    plan = G.GhostPlan(pool)
    dp = G.DevicePlan(plan, torch.device("cuda"))
    state = np.random.default_rng(1).standard_normal(pool.size)
    X = torch.from_numpy(state).cuda()
    Y = X.clone()
    lib = _lib.load()
    stream = torch.cuda.current_stream().cuda_stream
    wm = ctypes.cast(dp.wmid, ctypes.c_void_p)
    for _, dev, nops, npts in dp.fill:
        _lib.check(lib.bssn_b200_fill(stream, X.data_ptr(), dev.data_ptr(), nops, npts, wm))
        _lib.check(lib.bssn_b200_fill(stream, Y.data_ptr(), dev.data_ptr(), nops, npts + 5000, wm))
    assert torch.equal(X, Y)
    assert lib.bssn_b200_fill(stream, X.data_ptr(), dp.fill[0][1].data_ptr(), 0, 10, wm) == _lib.EINVAL


# ------------------------------------------------------------------ evolution
def _S(h, dt, t):
    from bssn3d_b200.fused_rhs import pack_S
    return pack_S(2.0, 0.06, dt, h, 0.6, 20.0, t, (1, 1, 1, 1), (1, 0), h, h)


def oracle_exchange_steps(pool, U, dt, nsteps, ko_sigma=0.1, ko_order=6, restrict=False):
    """The batched exchange step restated on the CPU: before each stage the
    stage input's ghosts are filled, each block's rate is taken on its
    padded array and only interiors are updated (evolve.py:125-137 per
    interior point), with enforcement after the last stage."""
    geo = A.geometry_of(pool)
    U = U.copy()
    bufs = {"U": U, "Ya": U.copy(), "Yb": U.copy()}
    ACC = np.zeros_like(U)
    t = 0.0
    for _ in range(nsteps):
        for s, (y, nxt) in enumerate([("U", "Ya"), ("Ya", "Yb"), ("Yb", "Ya"), ("Ya", "U")]):
            bufs[y][:] = A.fill(bufs[y], geo)
            cs = (0.0, 0.5, 0.5, 1.0)[s]
            for i, (G, blk) in enumerate(zip(geo, pool.blocks)):
                r = O.rate(G.view(bufs[y]), _S(blk.h, dt, t + cs * dt), ko_sigma, ko_order, ng=G.ng)
                I = (slice(None),) + (slice(G.ng, -G.ng),) * 3
                r = r[I]
                u = G.view(U)[I]
                acc = G.view(ACC)
                out = G.view(bufs[nxt])
                if s == 0:
                    acc[I] = r
                    out[I] = u + 0.5 * dt * r
                elif s < 3:
                    acc[I] = acc[I] + 2.0 * r
                    out[I] = u + (dt if s == 2 else 0.5 * dt) * r
                else:
                    out[I] = O.enforce(u + (dt / 6.0) * (acc[I] + r))
        if restrict:
            U[:] = A.restrict(U, geo)
        t += dt
    return U


@pytest.mark.parametrize("restrict", [False, True])
def test_exchange_rk4_steps_vs_oracle(restrict):
    from bssn3d_b200 import amr
    pool, punct = _pool(count=10, seed=7, domain=6.0, sizes=(8, 10, 12))
    U = pool.initial_state(punct, seed=2)
    dt = 0.25 * min(b.h for b in pool.blocks)
    evo = amr.BatchedEvolution(pool, ko_sigma=0.1, ko_order=6, variant=0, ghosts="exchange",
                               restrict=restrict)
    assert evo.plan.counts["copy"] > 0 and evo.plan.counts["prolong"] > 0
    got = evo.evolve(torch.from_numpy(U).cuda(), dt, 2).cpu().numpy()
    ref = oracle_exchange_steps(pool, U, dt, 2, restrict=restrict)
    assert np.isfinite(got).all()
    geo = A.geometry_of(pool)
    for i, G in enumerate(geo):
        I = (slice(None),) + (slice(G.ng, -G.ng),) * 3
        assert O.normwise_rel_grouped(G.view(got)[I], G.view(ref)[I]).max() < 1e-11, i


def test_exchange_variants_agree_and_rhs_fills_first():
    from bssn3d_b200 import amr
    pool, punct = _pool(count=10, seed=7, domain=6.0, sizes=(8, 10, 12))
    U = torch.from_numpy(pool.initial_state(punct, seed=2)).cuda()
    dt = 0.25 * min(b.h for b in pool.blocks)
    evo = amr.BatchedEvolution(pool, ko_sigma=0.1, ko_order=6, variant=0, ghosts="exchange")
    outs = []
    for v in range(4):
        evo.set_variant(v)
        outs.append(evo.evolve(U, dt, 1))
    for o in outs[1:]:
        assert torch.equal(o, outs[0])
    r = evo.rhs(U, evo.scalars(0.0, dt)).cpu().numpy()
    filled = A.fill(U.cpu().numpy(), A.geometry_of(pool))
    for i, (G, blk) in enumerate(zip(A.geometry_of(pool), pool.blocks)):
        I = (slice(None),) + (slice(G.ng, -G.ng),) * 3
        ref = O.rhs(G.view(filled), _S(blk.h, dt, 0.0))[I]
        # Where a rate is pure cancellation (chi's CAHD term on a block far from
        # the punctures is ~1e-8 of its terms) two correct evaluations differ by
        # more than 1e-12 of the result; the bar is then what the oracle and the
        # reference's compiled algebra themselves agree to.
        bar = np.full(24, 1e-12)
        if O.have_ref():
            other = O.ref_rhs(G.view(filled), _S(blk.h, dt, 0.0))[I]
            bar = np.maximum(bar, 4.0 * O.normwise_rel(ref, other))
        assert np.all(O.normwise_rel(G.view(r)[I], ref) <= bar), i


def test_workload_exchange_steps_stay_finite_with_constraint_norms():
    from bssn3d_b200 import amr
    blocks, punct, dt = amr.workload(3)
    pool = amr.BlockPool(blocks)
    U = torch.from_numpy(pool.initial_state(punct, seed=0)).cuda()
    evo = amr.BatchedEvolution(pool, ko_sigma=0.1, ko_order=6, variant=0, ghosts="exchange")
    h0, m0 = evo.constraint_norms(U)
    out = evo.evolve(U, dt, 2)
    assert bool(torch.isfinite(out).all())
    h1, m1 = evo.constraint_norms(out)
    assert np.isfinite([h0, m0, h1, m1]).all()
    assert h1 < 10 * h0 + 1.0


def test_distributed_evolution_one_rank_equals_batched_exchange():
    from bssn3d_b200 import amr
    from bssn3d_b200.parallel import DistributedBatchedEvolution
    pool, punct = _pool(count=10, seed=7, domain=6.0, sizes=(8, 10, 12))
    U = torch.from_numpy(pool.initial_state(punct, seed=2)).cuda()
    dt = 0.25 * min(b.h for b in pool.blocks)
    ref = amr.BatchedEvolution(pool, ko_sigma=0.1, ko_order=6, ghosts="exchange")
    dist_evo = DistributedBatchedEvolution(pool.blocks, world=1, rank=0, ko_sigma=0.1, ko_order=6)
    a = ref.evolve(U, dt, 2)
    b = dist_evo.evolve(U, dt, 2)
    assert torch.equal(a, b)
    assert dist_evo.constraint_norms(b) == ref.constraint_norms(a)
    # with restriction after every step
    ref_r = amr.BatchedEvolution(pool, ko_sigma=0.1, ko_order=6, ghosts="exchange", restrict=True)
    dist_r = DistributedBatchedEvolution(pool.blocks, world=1, rank=0, ko_sigma=0.1, ko_order=6, restrict=True)
    assert ref_r.plan.restrict_lists and dist_r.layout.restrict_levels
    assert torch.equal(ref_r.evolve(U, dt, 2), dist_r.evolve(U, dt, 2))
