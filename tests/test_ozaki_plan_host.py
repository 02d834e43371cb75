"""Host plan of the batched Ozaki calls (bssn_b200_batch_ozaki_plan), no GPU:
per pass kind the tile prefix over the blocks equals its restatement (128-line
groups x 16-output groups over the covered box), the point prefix counts the
covered interiors, and bad tables are refused."""

import ctypes

import pytest

KINDS = [(0, (0, 3, 3)), (0, (0, 0, 0)), (1, (0, 0, 3)), (1, (0, 0, 0)), (2, (0, 0, 0))]


def _tiles(shape, core, axis, ext):
    e = [s - 2 * max(core - x, 0) for s, x in zip(shape, ext)]
    nlines = e[(axis + 1) % 3] * e[(axis + 2) % 3]
    return -(-nlines // 128) * -(-e[axis] // 16)


def _pool():
    from bssn3d_b200 import amr
    from bssn3d_b200.initial_data import Puncture
    punct = [Puncture(0.909, (-0.5, 0.0, 0.0)), Puncture(0.0909, (1.0, 0.0, 0.0))]
    blocks = amr.nested_blocks(12, 3, punct, 6.0, 0.25, seed=5, sizes=(8, 16, 24), ng=3)
    return amr.BlockPool(blocks)


@pytest.mark.parametrize("core", [False, True])
def test_plan_matches_restatement(core):
    from bssn3d_b200.ozaki import ozaki_plan
    pool = _pool()
    table, _ = pool.descriptors(pool.tile, core=core)
    n = len(pool.blocks)
    tile0, ntiles, pts0, npts = ozaki_plan(table, n)
    for q, (axis, ext) in enumerate(KINDS):
        t = 0
        for b, blk in enumerate(pool.blocks):
            assert tile0[q * n + b] == t
            t += _tiles(blk.shape, blk.ng if core else 0, axis, ext)
        assert ntiles[q] == t
    want = pool.interior_points if core else pool.points
    assert npts == want
    c = 0
    for b, blk in enumerate(pool.blocks):
        assert pts0[b] == c
        c += blk.interior_points if core else blk.points


def test_plan_refuses_bad_tables():
    from bssn3d_b200 import _lib
    from bssn3d_b200.ozaki import ozaki_plan
    pool = _pool()
    table, _ = pool.descriptors(pool.tile, core=True)
    table[1].core = table[1].sx // 2
    with pytest.raises(_lib.BssnB200Error, match="core margin"):
        ozaki_plan(table, len(pool.blocks))
    table, _ = pool.descriptors(pool.tile, core=True)
    table[2].offset += 8
    with pytest.raises(_lib.BssnB200Error, match="offset"):
        ozaki_plan(table, len(pool.blocks))
    lib = _lib.load()
    assert lib.bssn_b200_batch_ozaki_plan(None, 0, None, None, None) == -1
