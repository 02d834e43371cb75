"""Multi-GPU layout of a batched block list: one process per GPU, each rank
evolves its own contiguous range of a Morton-ordered block list.

Blocks are independent units on this path (each carries its own ghosts), so
the ranks exchange nothing while they step; the only collectives are the
host-side barrier and the max-over-ranks timing reduction. Ranges are cut so
that every rank holds about the same cost (points per block, the fused
kernel's work is proportional to the padded volume).
"""

from __future__ import annotations

from typing import List, Sequence


def _morton3(ix: int, iy: int, iz: int, bits: int = 21) -> int:
    code = 0
    for b in range(bits):
        code |= ((ix >> b) & 1) << (3 * b + 2) | ((iy >> b) & 1) << (3 * b + 1) | ((iz >> b) & 1) << (3 * b)
    return code


def morton_order(blocks) -> List[int]:
    """Block indices sorted along a Z-order curve of the block origins."""
    hmin = min(b.h for b in blocks)
    lo = [min(b.origin[a] for b in blocks) for a in range(3)]
    keys = []
    for i, b in enumerate(blocks):
        q = [int(round((b.origin[a] - lo[a]) / hmin)) for a in range(3)]
        keys.append((_morton3(*q), i))
    return [i for _, i in sorted(keys)]


def partition(blocks: Sequence, world: int) -> List[List[int]]:
    """Contiguous ranges of the Morton order with balanced padded volume."""
    order = morton_order(blocks)
    total = sum(blocks[i].points for i in order)
    parts: List[List[int]] = [[] for _ in range(world)]
    acc, r = 0, 0
    for i in order:
        if r < world - 1 and acc >= total * (r + 1) / world:
            r += 1
        parts[r].append(i)
        acc += blocks[i].points
    return parts


def local_blocks(blocks: Sequence, rank: int, world: int):
    return [blocks[i] for i in partition(blocks, world)[rank]]
