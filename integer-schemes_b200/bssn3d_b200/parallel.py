"""Multi-GPU layout of a batched block list: one process per GPU, each rank
evolves its own contiguous range of a Morton-ordered block list.

With ghosts evolved in place (``ghosts="evolve"``) blocks are independent
units and the ranks exchange nothing while they step. With ghost exchange
(``ghosts="exchange"``) a block's ghosts come from other blocks, some owned by
other ranks: every rank computes the same global fill plan, keeps mirror
copies of the remote blocks its own ghosts read, and before each level's
fill receives those blocks from their owners (point-to-point, NCCL between
GPUs); the constraint norms take one all-reduce. Ranges are cut so that
every rank holds about the same cost (the fused kernel's work is
proportional to the padded volume).
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


class RankLayout:
    """What one rank holds for a ghost-exchanging block list.

    ``index``: global indices of the blocks in this rank's pool, ascending —
    its own blocks (``owned``, positions in the pool) and mirrors of the
    remote blocks its ghost fill reads. ``fill_lists``: the global plan's
    ops whose destination this rank owns, remapped to the local pool.
    ``recv[level]`` / ``send[level]``: [(peer rank, global block)] moved
    before that level's fill, in global block order (both sides post their
    messages for a peer in the same order, so they pair up).
    """

    def __init__(self, blocks: Sequence, world: int, rank: int, plan=None):
        import ctypes as _ct
        from .amr import BlockPool
        from .ghosts import FillOp, GhostPlan
        self.world, self.rank = int(world), int(rank)
        self.parts = partition(blocks, world)
        owner = {}
        for r, part in enumerate(self.parts):
            for i in part:
                owner[i] = r
        gpool = BlockPool(blocks)
        gplan = plan if plan is not None else GhostPlan(gpool)
        if gplan.restrict_lists:
            raise ValueError("restriction across ranks is not provided: build the plan without it")
        off2idx = {int(o): i for i, o in enumerate(gpool.offsets)}
        # for every rank: the remote sources its own ghost boxes read, per level
        needs = {r: {} for r in range(world)}
        per_rank_ops = {r: [] for r in range(world)}
        for lvl, ops in gplan.fill_lists:
            for r in range(world):
                keep = [op for op in ops if owner[off2idx[op.dst_off]] == r]
                per_rank_ops[r].append((lvl, keep))
                needs[r][lvl] = sorted({off2idx[op.src_off] for op in keep if owner[off2idx[op.src_off]] != r})
        mirrors = sorted({j for v in needs[rank].values() for j in v})
        self.index = sorted(set(self.parts[rank]) | set(mirrors))
        g2l = {g: l for l, g in enumerate(self.index)}
        self.owned = sorted(g2l[g] for g in self.parts[rank])
        self.pool = BlockPool([blocks[i] for i in self.index])
        self.fill_lists = []
        for lvl, keep in per_rank_ops[rank]:
            local = []
            for op in keep:
                q = FillOp()
                _ct.pointer(q)[0] = op
                q.dst_off = int(self.pool.offsets[g2l[off2idx[op.dst_off]]])
                q.src_off = int(self.pool.offsets[g2l[off2idx[op.src_off]]])
                local.append(q)
            if local:
                self.fill_lists.append((lvl, local))
        self.restrict_lists = []
        self.levels = [lvl for lvl, _ in gplan.fill_lists]
        self.recv = {lvl: [(owner[j], j) for j in needs[rank][lvl]] for lvl in self.levels}
        self.send = {lvl: sorted(((q, j) for q in range(world) if q != rank
                                  for j in needs[q][lvl] if owner[j] == rank), key=lambda t: (t[1], t[0]))
                     for lvl in self.levels}
        self.recv = {lvl: sorted(v, key=lambda t: (t[1], t[0])) for lvl, v in self.recv.items()}
        self.g2l = g2l

    def block_view(self, pool_tensor, g: int):
        """The flat view of global block ``g`` in this rank's pool tensor."""
        i = self.g2l[g]
        o = int(self.pool.offsets[i])
        return pool_tensor[o:o + 24 * self.pool.blocks[i].points]

    def exchange(self, pool_tensor, level: int, group=None) -> None:
        """Move the blocks the ``level`` fill reads across ranks: send this
        rank's blocks that others mirror, receive its own mirrors."""
        import torch.distributed as dist
        if self.world == 1:
            return
        ops = []
        for q, j in self.send.get(level, []):
            ops.append(dist.P2POp(dist.isend, self.block_view(pool_tensor, j), q, group=group))
        for p, j in self.recv.get(level, []):
            ops.append(dist.P2POp(dist.irecv, self.block_view(pool_tensor, j), p, group=group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()


class DistributedBatchedEvolution:
    """RK4 over a block list split across ranks, ghosts exchanged each stage:
    per stage, per level from coarse to fine, the mirrors this rank's fill
    reads are received from their owners, then the level's fill boxes run
    (``bssn_b200_fill``), then one batched stage launch evolves this rank's
    own blocks. Eager (not graph-captured: the point-to-point transfers sit
    between the launches). ``world == 1`` is the single-GPU exchange path."""

    def __init__(self, blocks: Sequence, punctures=None, world: int = 1, rank: int = 0, ko_sigma: float = 0.1,
                 ko_order: int = 6, variant: int = 0, device="cuda", group=None):
        from .amr import BatchedEvolution
        self.layout = RankLayout(blocks, world, rank)
        self.group = group
        self.evo = BatchedEvolution(self.layout.pool, ko_sigma=ko_sigma, ko_order=ko_order, variant=variant,
                                    device=device, ghosts="exchange", plan=self.layout,
                                    active=self.layout.owned)

    def fill(self, Y) -> None:
        stream = self.evo._stream()
        for lvl in self.layout.levels:
            self.layout.exchange(Y, lvl, self.group)
            self.evo.dplan.run_level("fill", lvl, Y, stream)

    def step_inplace(self, U, S) -> None:
        b = self.evo.buffers(U)
        for stage, (y, ynext) in enumerate([(U, b["Ya"]), (b["Ya"], b["Yb"]), (b["Yb"], b["Ya"]),
                                            (b["Ya"], U)]):
            self.fill(y)
            self.evo.stage(stage, U, y, b["ACC"], ynext, S)

    def evolve(self, U, dt: float, nsteps: int, t0: float = 0.0):
        U = U.clone()
        self.evo.seed_buffers(U)
        S = self.evo.scalars(t0, dt)
        for _ in range(int(nsteps)):
            self.step_inplace(U, S)
            self.evo.advance_time(S)
        return U

    def constraint_norms(self, U):
        """Interior norms (H, |M|) over every rank's own blocks together (one all-reduce)."""
        import torch
        Y = U.clone()
        self.fill(Y)
        sums = self.evo.constraint_sums(Y, filled=True)
        if self.layout.world > 1:
            import torch.distributed as dist
            dist.all_reduce(sums, group=self.group)
        hm = torch.sqrt(sums[:2] / sums[2])
        return float(hm[0]), float(hm[1])
