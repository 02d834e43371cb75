"""Ghost-exchange plan of the batched AMR path, checked on the CPU.

The box planner (bssn3d_b200.ghosts) must give every ghost point the source
the oracle picks point by point from the geometry, and its boxes, executed
here with numpy, must reproduce the oracle's fill and restriction exactly.
The transfer operators themselves are checked for the properties the
reference tests (3D/tests/multipatch_amr/test_transfer.py:24-90)."""

import ctypes
import itertools

import numpy as np
import pytest

from oracle import amr_oracle as A


def small_pool(seed=7, count=14, ng=3):
    from bssn3d_b200 import amr
    from bssn3d_b200.initial_data import Puncture
    punct = [Puncture(0.909, (-0.5, 0.0, 0.0)), Puncture(0.0909, (1.0, 0.0, 0.0))]
    blocks = amr.nested_blocks(count, 3, punct, 4.0, 0.25, seed=seed, sizes=(6, 8, 10),
                               probs=(0.4, 0.4, 0.2), ng=ng)
    return amr.BlockPool(blocks)


def octree_pool(corner, BS=16, NG=4):
    """One parent (level 0, h = 1) and one child in octant ``corner``."""
    from bssn3d_b200 import amr
    parent = amr.Block(level=0, n=BS, origin=(0.0, 0.0, 0.0), h=1.0, ng=NG)
    child = amr.Block(level=1, n=BS, origin=tuple(c * BS / 2 for c in corner), h=0.5, ng=NG)
    return amr.BlockPool([parent, child])


def execute(pool, plan, state, which="fill"):
    """Run the plan's boxes with numpy (list by list, in order)."""
    from bssn3d_b200 import ghosts as G
    out = state.copy()
    geo = A.geometry_of(pool)
    by_off = {g.offset: g for g in geo}
    lists = plan.fill_lists if which == "fill" else plan.restrict_lists
    for _, ops in lists:
        snap = out.copy()   # one launch: every box reads the pool as it was
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
            D.view(out)[:, d[:, 0], d[:, 1], d[:, 2]] = val
    return out


# ------------------------------------------------------------------ box algebra
def test_subtract_and_intersect_partition_a_box():
    from bssn3d_b200.ghosts import intersect, subtract, volume
    rng = np.random.default_rng(0)
    for _ in range(200):
        lo = rng.integers(-4, 4, 6)
        a = (lo[0], lo[1], lo[2], lo[0] + rng.integers(1, 6), lo[1] + rng.integers(1, 6), lo[2] + rng.integers(1, 6))
        lo = rng.integers(-4, 4, 3)
        b = (lo[0], lo[1], lo[2], lo[0] + rng.integers(1, 6), lo[1] + rng.integers(1, 6), lo[2] + rng.integers(1, 6))
        a = tuple(int(v) for v in a)
        b = tuple(int(v) for v in b)
        grid = np.zeros((16, 16, 16), int)
        c = intersect(a, b)
        pieces = [a] if c is None else subtract(a, c)
        for p in pieces:
            grid[p[0] + 8:p[3] + 8, p[1] + 8:p[4] + 8, p[2] + 8:p[5] + 8] += 1
        want = np.zeros_like(grid)
        want[a[0] + 8:a[3] + 8, a[1] + 8:a[4] + 8, a[2] + 8:a[5] + 8] = 1
        if c is not None:
            want[c[0] + 8:c[3] + 8, c[1] + 8:c[4] + 8, c[2] + 8:c[5] + 8] = 0
            assert volume(c) + sum(volume(p) for p in pieces) == volume(a)
        assert np.array_equal(grid, want)


def test_midpoint_weights():
    from bssn3d_b200.ghosts import W_MID
    assert np.array_equal(W_MID, A.W)
    np.testing.assert_allclose(W_MID * 256, [3, -25, 150, 150, -25, 3], rtol=0, atol=1e-12)
    assert abs(W_MID.sum() - 1.0) < 1e-15


# ------------------------------------------------------------------ planner
@pytest.mark.parametrize("seed", [7, 11])
def test_plan_sources_match_oracle_point_by_point(seed):
    from bssn3d_b200 import ghosts as G
    pool = small_pool(seed)
    plan = G.GhostPlan(pool)
    geo = A.geometry_of(pool)
    by_off = {g.offset: i for i, g in enumerate(geo)}
    got = {}
    for lvl, ops in plan.fill_lists:
        for op in ops:
            b, s = by_off[op.dst_off], by_off[op.src_off]
            assert geo[b].level == lvl
            d = np.indices([op.hi[k] - op.lo[k] for k in range(3)]).reshape(3, -1).T + list(op.lo)
            ng, S = geo[b].ng, geo[b].S
            assert not np.any(np.all((d >= ng) & (d < S - ng), axis=1)), "a box writes an interior point"
            for p in map(tuple, d):
                assert (b, p) not in got, "two boxes write one point"
                got[(b, p)] = (op.kind, s)
    kinds = set()
    for b in range(len(geo)):
        loc, kind, src = A.sources(geo, b)
        for p, k, s in zip(map(tuple, loc), kind, src):
            if k < 0:
                assert (b, p) not in got
            else:
                assert got[(b, p)] == (k, s)
                kinds.add(int(k))
    assert kinds == {G.COPY, G.PROLONG}
    total = sum(plan.counts.values())
    assert total == sum(int(np.prod(g.S)) - (int(g.S[0]) - 2 * g.ng) ** 3 for g in geo)


def test_plan_execution_equals_oracle_fill_and_restriction():
    from bssn3d_b200 import ghosts as G
    pool = small_pool(11)
    plan = G.GhostPlan(pool, restrict=True)
    assert plan.restrict_lists
    geo = A.geometry_of(pool)
    state = np.random.default_rng(3).standard_normal(pool.size)
    assert np.array_equal(execute(pool, plan, state), A.fill(state, geo))
    assert np.array_equal(execute(pool, plan, state, "restrict"), A.restrict(state, geo))


def test_device_table_layout_and_c_validation():
    from bssn3d_b200 import _lib, ghosts as G
    assert ctypes.sizeof(G.FillOp) == 88
    pool = small_pool(7)
    plan = G.GhostPlan(pool)
    lib = _lib.load()
    for _, ops in plan.fill_lists:
        arr = (G.FillOp * len(ops))(*ops)
        total = lib.bssn_b200_fill_plan(ctypes.addressof(arr), len(ops), pool.size)
        vols = [(o.hi[0] - o.lo[0]) * (o.hi[1] - o.lo[1]) * (o.hi[2] - o.lo[2]) for o in arr]
        assert total == sum(vols)
        assert [a.point0 for a in arr] == list(np.cumsum([0] + vols[:-1]))
        kinds = [a.kind for a in arr]   # copies and injections first, prolongations after, stable
        assert kinds == sorted(kinds, key=lambda k: k == G.PROLONG)
        key = lambda o: (o.dst_off, o.src_off, tuple(o.lo), tuple(o.hi), o.kind)
        assert sorted(map(key, arr)) == sorted(map(key, ops))
        assert [key(a) for a in arr if a.kind != G.PROLONG] == [key(o) for o in ops if o.kind != G.PROLONG]
    ops = plan.fill_lists[-1][1]
    bad = [(lambda o: setattr(o, "kind", 7), "kind"),
           (lambda o: o.hi.__setitem__(0, o.dst_s[0] + 1), "box"),
           (lambda o: setattr(o, "dst_off", pool.size), "pool"),
           (lambda o: setattr(o, "src_off", o.dst_off), "itself")]
    for mutate, word in bad:
        arr = (G.FillOp * len(ops))(*ops)
        mutate(arr[0])
        assert lib.bssn_b200_fill_plan(ctypes.addressof(arr), len(ops), pool.size) == -1
        assert word in lib.bssn_b200_last_error().decode()
    copy = next(o for o in ops if o.kind == G.COPY)
    arr = (G.FillOp * 1)(copy)
    arr[0].shift[2] += 100
    assert lib.bssn_b200_fill_plan(ctypes.addressof(arr), 1, pool.size) == -1
    assert "source" in lib.bssn_b200_last_error().decode()


def test_core_descriptors_agree_with_c_planner():
    from bssn3d_b200 import _lib
    pool = small_pool(7)
    lib = _lib.load()
    ref, tiles = pool.descriptors((4, 4, 16), core=True)
    table, _ = pool.descriptors((4, 4, 16), core=True)
    assert all(t.core == b.ng for t, b in zip(table, pool.blocks))
    assert lib.bssn_b200_batch_plan(ctypes.addressof(table), len(pool.blocks), 0) == tiles
    assert [t.tile0 for t in table] == [t.tile0 for t in ref]
    table[0].core = table[0].sx // 2
    assert lib.bssn_b200_batch_plan(ctypes.addressof(table), len(pool.blocks), 0) == -1


def test_octree_child_halo_is_the_cropped_refined_parent():
    """The reference's sync_across_levels: the child's whole halo is the
    parent, refined, cropped at NG + corner*BS (kernels.py:76-102)."""
    from bssn3d_b200 import ghosts as G
    BS, NG = 16, 4
    for corner in [(0, 0, 0), (1, 0, 1), (1, 1, 1)]:
        pool = octree_pool(corner, BS, NG)
        plan = G.GhostPlan(pool)
        state = np.random.default_rng(2).standard_normal(pool.size)
        out = execute(pool, plan, state)
        geo = A.geometry_of(pool)
        s = [NG + c * BS for c in corner]
        W = BS + 2 * NG
        want = A.refine(geo[0].view(state))[:, s[0]:s[0] + W, s[1]:s[1] + W, s[2]:s[2] + W]
        child = geo[1].view(out)
        halo = np.ones((W, W, W), bool)
        halo[NG:NG + BS, NG:NG + BS, NG:NG + BS] = False
        assert np.array_equal(child[:, halo], want[:, halo])
        assert np.array_equal(child[:, ~halo], geo[1].view(state)[:, ~halo])


# ------------------------------------------------------------------ operators
@pytest.mark.parametrize("corner", list(itertools.product((0, 1), repeat=3)))
def test_coincident_nodes_copy_exactly(corner):
    BS, NG = 16, 4
    parent = np.random.default_rng(0).standard_normal((24,) + (BS + 2 * NG,) * 3)
    r = A.refine(parent)
    half = BS // 2
    a = np.arange(half)
    # refined index of parent node q is 2q
    fx = 2 * (NG + corner[0] * half + a)
    fy = 2 * (NG + corner[1] * half + a)
    fz = 2 * (NG + corner[2] * half + a)
    got = r[np.ix_(np.arange(24), fx, fy, fz)]
    px = NG + corner[0] * half + a
    py = NG + corner[1] * half + a
    pz = NG + corner[2] * half + a
    assert np.array_equal(got, parent[np.ix_(np.arange(24), px, py, pz)])


def test_degree_five_polynomials_are_reproduced():
    BS, NG, h = 16, 4, 0.37
    W = BS + 2 * NG
    cx = np.array([0.4, -1.1, 0.7, 0.2, -0.3, 0.15])
    cy = np.array([-0.5, 0.9, -0.2, 0.6, 0.1, -0.25])
    cz = np.array([0.8, 0.3, -0.6, -0.1, 0.45, 0.05])
    P = lambda c, x: sum(c[d] * x ** d for d in range(6))
    xp = (np.arange(W) - NG) * h
    parent = np.einsum("i,j,k->ijk", P(cx, xp), P(cy, xp), P(cz, xp))[None].repeat(2, 0)
    r = A.refine(parent)
    # child (corner 0) index ff sits at refined index NG + ff, coordinate (ff - NG) h / 2
    ff = np.arange(NG + 3, NG + BS - 3)
    xf = (ff - NG) * h / 2
    want = np.einsum("i,j,k->ijk", P(cx, xf), P(cy, xf), P(cz, xf))
    g = NG + ff
    assert np.max(np.abs(r[np.ix_([0, 1], g, g, g)] - want[None])) < 1e-9


def test_restriction_inverts_prolongation():
    from bssn3d_b200 import ghosts as G
    BS, NG = 16, 4
    for corner in [(0, 1, 0), (1, 1, 0)]:
        pool = octree_pool(corner, BS, NG)
        geo = A.geometry_of(pool)
        state = np.random.default_rng(5).standard_normal(pool.size)
        s = [NG + c * BS for c in corner]
        W = BS + 2 * NG
        geo[1].view(state)[:] = A.refine(geo[0].view(state))[:, s[0]:s[0] + W, s[1]:s[1] + W, s[2]:s[2] + W]
        parent_before = geo[0].view(state).copy()
        geo[0].view(state)[:, NG:NG + BS, NG:NG + BS, NG:NG + BS] = 0.0
        plan = G.GhostPlan(pool, restrict=True)
        out = execute(pool, plan, state, "restrict")
        half = BS // 2
        sl = tuple(slice(NG + c * half, NG + c * half + half) for c in corner)
        assert np.array_equal(geo[0].view(out)[(slice(None),) + sl], parent_before[(slice(None),) + sl])
