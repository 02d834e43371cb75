"""Multi-GPU layout of a batched block list: one process per GPU, each rank
evolves its own contiguous range of a Morton-ordered block list.

With ghosts evolved in place (``ghosts="evolve"``) blocks are independent
units and the ranks exchange nothing while they step. With ghost exchange
(``ghosts="exchange"``) a block's ghosts come from other blocks, some owned by
other ranks: every rank computes the same global fill plan, keeps mirror
copies of the remote blocks its own ghosts read, and before each level's
fill receives those blocks from their owners (point-to-point, NCCL between
GPUs) — only the points its fill boxes read, gathered into one buffer per
peer and level (whole mirrored blocks are the fallback); the constraint
norms take one all-reduce. Ranges are cut so that
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


def read_box(op):
    """The box of source-block points a fill op reads, half-open per axis
    ((lo, hi) x 3), clamped to the source array: the shifted destination box
    for a same-level copy; for a prolongation, the source nodes of every
    refined index g = d + shift (node g/2 for even g, the six nodes
    (g-1)/2 - 2 ... (g-1)/2 + 3 for odd g). Restriction ops are not read
    across ranks."""
    from .ghosts import COPY, PROLONG
    box = []
    for a in range(3):
        s = op.src_s[a]
        gmin, gmax = op.lo[a] + op.shift[a], op.hi[a] - 1 + op.shift[a]
        if op.kind == COPY:
            lo, hi = gmin, gmax + 1
        elif op.kind == PROLONG:
            lo, hi = (gmin - 1) // 2 - 2, (gmax - 1) // 2 + 3 + 1
        else:
            raise ValueError("restriction ops are not exchanged across ranks")
        box.append((max(lo, 0), min(hi, s)))
    return box


def box_points(box, shape) -> "np.ndarray":
    """Flat in-block indices (C order) of the points of ``box``."""
    import numpy as np
    (x0, x1), (y0, y1), (z0, z1) = box
    sy, sz = shape[1], shape[2]
    x, y, z = np.meshgrid(np.arange(x0, x1), np.arange(y0, y1), np.arange(z0, z1), indexing="ij")
    return ((x * sy + y) * sz + z).reshape(-1).astype(np.int64)


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
        # Packed halos: the points of a remote block that a rank's fill reads
        # at a level (the union of its ops' read boxes), so that only those
        # cross between ranks instead of whole block arrays.
        import numpy as np
        reads = {r: {} for r in range(world)}   # r -> {(lvl, j): point indices}
        for r in range(world):
            for lvl, keep in per_rank_ops[r]:
                for op in keep:
                    j = off2idx[op.src_off]
                    if owner[j] == r:
                        continue
                    pts = box_points(read_box(op), blocks[j].shape)
                    key = (lvl, j)
                    reads[r][key] = pts if key not in reads[r] else np.union1d(reads[r][key], pts)
        self._reads = reads
        self._packed = {}

    def _pack_index(self, pairs, points_of):
        """Flat pool indices (24 fields x points, block by block in the given
        order) of the packed points of ``pairs`` [(peer, global block)]."""
        import numpy as np
        parts = []
        for _, j in pairs:
            pts = points_of(j)
            i = self.g2l[j]
            o, n = int(self.pool.offsets[i]), self.pool.blocks[i].points
            parts.append((o + np.arange(24, dtype=np.int64)[:, None] * n + pts[None, :]).reshape(-1))
        return np.concatenate(parts) if parts else np.zeros(0, dtype=np.int64)

    def packed_plan(self, device):
        """Per level and peer, the device index lists of the packed exchange:
        {level: ([(peer, send index)], [(peer, recv index)])}, messages in
        global block order (both sides build them from the same global plan)."""
        import torch
        key = str(device)
        if key in self._packed:
            return self._packed[key]
        plan = {}
        for lvl in self.levels:
            sends, recvs = [], []
            for q in range(self.world):
                sp = [(q2, j) for q2, j in self.send.get(lvl, []) if q2 == q]
                if sp:
                    idx = self._pack_index(sp, lambda j, q=q: self._reads[q][(lvl, j)])
                    sends.append((q, torch.from_numpy(idx).to(device)))
                rp = [(p, j) for p, j in self.recv.get(lvl, []) if p == q]
                if rp:
                    idx = self._pack_index(rp, lambda j: self._reads[self.rank][(lvl, j)])
                    recvs.append((q, torch.from_numpy(idx).to(device)))
            plan[lvl] = (sends, recvs)
        self._packed[key] = plan
        return plan

    def exchange_bytes(self, packed: bool = True) -> int:
        """Bytes this rank sends per fill (all levels), packed or whole blocks."""
        total = 0
        for lvl in self.levels:
            for q, j in self.send.get(lvl, []):
                total += 8 * 24 * (len(self._reads[q][(lvl, j)]) if packed else self.pool.blocks[self.g2l[j]].points)
        return total

    def exchange_packed(self, pool_tensor, level: int, group=None) -> None:
        """:meth:`exchange` moving only the points the receivers' fill boxes
        read: one gathered buffer per peer and level each way, scattered into
        the mirrors on arrival. Mirror points outside the read boxes are not
        kept up to date (no fill box reads them)."""
        import torch
        import torch.distributed as dist
        if self.world == 1:
            return
        sends, recvs = self.packed_plan(pool_tensor.device)[level]
        flat = pool_tensor.view(-1)
        ops, bufs = [], []
        for q, idx in sends:
            ops.append(dist.P2POp(dist.isend, flat[idx], q, group=group))
        for p, idx in recvs:
            buf = torch.empty(idx.numel(), dtype=pool_tensor.dtype, device=pool_tensor.device)
            bufs.append((idx, buf))
            ops.append(dist.P2POp(dist.irecv, buf, p, group=group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        for idx, buf in bufs:
            flat[idx] = buf

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
    per stage, per level from coarse to fine, the points of remote blocks this
    rank's fill reads are received from their owners (packed; whole blocks
    with ``packed=False``), then the level's fill boxes run
    (``bssn_b200_fill``), then one batched stage launch evolves this rank's
    own blocks. Eager (not graph-captured: the point-to-point transfers sit
    between the launches). ``world == 1`` is the single-GPU exchange path."""

    def __init__(self, blocks: Sequence, punctures=None, world: int = 1, rank: int = 0, ko_sigma: float = 0.1,
                 ko_order: int = 6, variant: int = 0, device="cuda", group=None, packed: bool = True):
        from .amr import BatchedEvolution
        self.layout = RankLayout(blocks, world, rank)
        self.group = group
        self.packed = bool(packed)
        self.evo = BatchedEvolution(self.layout.pool, ko_sigma=ko_sigma, ko_order=ko_order, variant=variant,
                                    device=device, ghosts="exchange", plan=self.layout,
                                    active=self.layout.owned)

    def fill(self, Y) -> None:
        stream = self.evo._stream()
        for lvl in self.layout.levels:
            if self.packed:
                self.layout.exchange_packed(Y, lvl, self.group)
            else:
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
