"""Multi-GPU layout of a batched block list: one process per GPU, each rank
evolves its own contiguous range of a Morton-ordered block list.

With ghosts evolved in place (``ghosts="evolve"``) blocks are independent
units and the ranks exchange nothing while they step. With ghost exchange
(``ghosts="exchange"``) a block's ghosts come from other blocks, some owned by
other ranks: every rank computes the same global fill plan, keeps mirror
copies of the remote blocks its own ghosts read, and before each level's
fill receives those blocks from their owners (point-to-point, NCCL between
GPUs) — only the points its fill boxes read, gathered into one buffer per
peer and level (whole mirrored blocks are the fallback); the optional
restriction after a step receives the remote fine points it injects the same
way, finest level first; the constraint norms take one all-reduce. Ranges
are cut so that
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
    (g-1)/2 - 2 ... (g-1)/2 + 3 for odd g); for an injection the box spanned
    by 2 d + shift (it reads every other point of it, see :func:`read_points`)."""
    from .ghosts import COPY, PROLONG, RESTRICT
    box = []
    for a in range(3):
        s = op.src_s[a]
        gmin, gmax = op.lo[a] + op.shift[a], op.hi[a] - 1 + op.shift[a]
        if op.kind == COPY:
            lo, hi = gmin, gmax + 1
        elif op.kind == PROLONG:
            lo, hi = (gmin - 1) // 2 - 2, (gmax - 1) // 2 + 3 + 1
        elif op.kind == RESTRICT:
            lo, hi = 2 * op.lo[a] + op.shift[a], 2 * (op.hi[a] - 1) + op.shift[a] + 1
        else:
            raise ValueError(f"unknown fill kind {op.kind}")
        box.append((max(lo, 0), min(hi, s)))
    return box


def read_points(op, shape) -> "np.ndarray":
    """Flat in-block indices of the source points an op reads: its read box,
    or for an injection (src[2 d + shift]) every other point of it."""
    import numpy as np
    from .ghosts import RESTRICT
    if op.kind != RESTRICT:
        return box_points(read_box(op), shape)
    ax = [2 * np.arange(op.lo[a], op.hi[a]) + op.shift[a] for a in range(3)]
    x, y, z = np.meshgrid(*ax, indexing="ij")
    return ((x * shape[1] + y) * shape[2] + z).reshape(-1).astype(np.int64)


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
        import numpy as np
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
        off2idx = {int(o): i for i, o in enumerate(gpool.offsets)}
        # Per phase (ghost fill; restriction): the ops each rank runs (those
        # whose destination it owns), the remote source blocks they read, and
        # the exact source points read (the union of the ops' read points).
        phases = {"fill": gplan.fill_lists, "restrict": gplan.restrict_lists}
        per_rank_ops = {ph: {r: [] for r in range(world)} for ph in phases}
        needs = {ph: {r: {} for r in range(world)} for ph in phases}
        reads = {ph: {r: {} for r in range(world)} for ph in phases}
        for ph, lists in phases.items():
            for lvl, ops in lists:
                for r in range(world):
                    keep = [op for op in ops if owner[off2idx[op.dst_off]] == r]
                    per_rank_ops[ph][r].append((lvl, keep))
                    needs[ph][r][lvl] = sorted({off2idx[op.src_off] for op in keep
                                                if owner[off2idx[op.src_off]] != r})
                    for op in keep:
                        j = off2idx[op.src_off]
                        if owner[j] == r:
                            continue
                        pts = read_points(op, blocks[j].shape)
                        key = (lvl, j)
                        got = reads[ph][r].get(key)
                        reads[ph][r][key] = pts if got is None else np.union1d(got, pts)
        mirrors = sorted({j for ph in phases for v in needs[ph][rank].values() for j in v})
        self.index = sorted(set(self.parts[rank]) | set(mirrors))
        g2l = {g: l for l, g in enumerate(self.index)}
        self.g2l = g2l
        self.owned = sorted(g2l[g] for g in self.parts[rank])
        self.pool = BlockPool([blocks[i] for i in self.index])

        def local_lists(ph):
            out = []
            for lvl, keep in per_rank_ops[ph][rank]:
                local = []
                for op in keep:
                    q = FillOp()
                    _ct.pointer(q)[0] = op
                    q.dst_off = int(self.pool.offsets[g2l[off2idx[op.dst_off]]])
                    q.src_off = int(self.pool.offsets[g2l[off2idx[op.src_off]]])
                    local.append(q)
                if local:
                    out.append((lvl, local))
            return out

        def pairs(ph):
            levels = [lvl for lvl, _ in phases[ph]]
            recv = {lvl: sorted(((owner[j], j) for j in needs[ph][rank][lvl]), key=lambda t: (t[1], t[0]))
                    for lvl in levels}
            send = {lvl: sorted(((q, j) for q in range(world) if q != rank
                                 for j in needs[ph][q][lvl] if owner[j] == rank), key=lambda t: (t[1], t[0]))
                    for lvl in levels}
            return levels, send, recv

        self.fill_lists = local_lists("fill")
        self.restrict_lists = local_lists("restrict")
        self.levels, self.send, self.recv = pairs("fill")
        self.restrict_levels, self.send_restrict, self.recv_restrict = pairs("restrict")
        self._reads = reads["fill"]
        self._reads_restrict = reads["restrict"]
        self._packed = {}

    def _phase(self, phase: str):
        if phase == "fill":
            return self.levels, self.send, self.recv, self._reads
        if phase == "restrict":
            return self.restrict_levels, self.send_restrict, self.recv_restrict, self._reads_restrict
        raise ValueError(f"phase must be 'fill' or 'restrict', not {phase!r}")

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

    def packed_plan(self, device, phase: str = "fill"):
        """Per level and peer, the device index lists of a phase's packed
        exchange: {level: ([(peer, send index)], [(peer, recv index)])},
        messages in global block order (both sides build them from the same
        global plan)."""
        import torch
        key = (str(device), phase)
        if key in self._packed:
            return self._packed[key]
        levels, send, recv, reads = self._phase(phase)
        plan = {}
        for lvl in levels:
            sends, recvs = [], []
            for q in range(self.world):
                sp = [(q2, j) for q2, j in send.get(lvl, []) if q2 == q]
                if sp:
                    idx = self._pack_index(sp, lambda j, q=q: reads[q][(lvl, j)])
                    sends.append((q, torch.from_numpy(idx).to(device)))
                rp = [(p, j) for p, j in recv.get(lvl, []) if p == q]
                if rp:
                    idx = self._pack_index(rp, lambda j: reads[self.rank][(lvl, j)])
                    recvs.append((q, torch.from_numpy(idx).to(device)))
            plan[lvl] = (sends, recvs)
        self._packed[key] = plan
        return plan

    def exchange_bytes(self, packed: bool = True, phase: str = "fill") -> int:
        """Bytes this rank sends per pass of a phase (all levels), packed or
        whole blocks."""
        levels, send, _, reads = self._phase(phase)
        total = 0
        for lvl in levels:
            for q, j in send.get(lvl, []):
                total += 8 * 24 * (len(reads[q][(lvl, j)]) if packed else self.pool.blocks[self.g2l[j]].points)
        return total

    def exchange_packed(self, pool_tensor, level: int, group=None, phase: str = "fill") -> None:
        """:meth:`exchange` moving only the points the receivers' boxes read:
        one gathered buffer per peer and level each way, scattered into the
        mirrors on arrival. Mirror points outside the read boxes are not kept
        up to date (no box reads them)."""
        import torch
        import torch.distributed as dist
        if self.world == 1:
            return
        sends, recvs = self.packed_plan(pool_tensor.device, phase)[level]
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

    def exchange(self, pool_tensor, level: int, group=None, phase: str = "fill") -> None:
        """Move the blocks a phase's ``level`` boxes read across ranks: send
        this rank's blocks that others mirror, receive its own mirrors."""
        import torch.distributed as dist
        if self.world == 1:
            return
        _, send, recv, _ = self._phase(phase)
        ops = []
        for q, j in send.get(level, []):
            ops.append(dist.P2POp(dist.isend, self.block_view(pool_tensor, j), q, group=group))
        for p, j in recv.get(level, []):
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
                 ko_order: int = 6, variant: int = 0, device="cuda", group=None, packed: bool = True,
                 restrict: bool = False):
        from .amr import BatchedEvolution, BlockPool
        from .ghosts import GhostPlan
        self.layout = RankLayout(blocks, world, rank, plan=GhostPlan(BlockPool(blocks), restrict=restrict))
        self.group = group
        self.packed = bool(packed)
        self.evo = BatchedEvolution(self.layout.pool, ko_sigma=ko_sigma, ko_order=ko_order, variant=variant,
                                    device=device, ghosts="exchange", plan=self.layout,
                                    active=self.layout.owned)

    def _run(self, phase: str, levels, Y) -> None:
        stream = self.evo._stream()
        for lvl in levels:
            if self.packed:
                self.layout.exchange_packed(Y, lvl, self.group, phase=phase)
            else:
                self.layout.exchange(Y, lvl, self.group, phase=phase)
            self.evo.dplan.run_level(phase, lvl, Y, stream)

    def fill(self, Y) -> None:
        """Ghost fill of Y, coarse level first, remote sources received per level."""
        self._run("fill", self.layout.levels, Y)

    def restrict(self, U) -> None:
        """Injection of fine interiors into the coarser levels, finest first,
        remote fine points received per level (``restrict=True``)."""
        self._run("restrict", self.layout.restrict_levels, U)

    def step_inplace(self, U, S) -> None:
        b = self.evo.buffers(U)
        for stage, (y, ynext) in enumerate([(U, b["Ya"]), (b["Ya"], b["Yb"]), (b["Yb"], b["Ya"]),
                                            (b["Ya"], U)]):
            self.fill(y)
            self.evo.stage(stage, U, y, b["ACC"], ynext, S)
        if self.layout.restrict_levels:
            self.restrict(U)

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
