"""Ghost-zone exchange plan for a BSSN block pool (``bssn_b200_fill``).

The reference fills AMR ghosts in 3D/src/multipatch/amr/sync.py: each fine
block's halo is prolongated from its parent (``sync_across_levels``, :70-88),
then same-level neighbours overwrite what they hold exactly
(``sync_within_level``, :105-122); restriction injects fine interiors into
the coarse level (kernels.py:114-145). The operators are node-centred 2:1:
coincident nodes copy, midpoints take the 6-point Lagrange stencil at +1/2
(kernels.py:36-71), with the parent's array edge-padded.

Blocks here are cubes of mixed sizes on nested levels, not octants of one
parent, so the plan is built from the lattice geometry. Every block sits on
its level's node lattice (spacing h_l = h_0 / 2^l, nodes at integer
multiples of h_l, so the coarse lattice is every second fine node). For each
block, level by level from coarse to fine, its ghost shell (six slabs) is cut
into boxes, each with exactly one source:

1. COPY from the first same-level block (in pool order) whose interior holds
   the points: exact data wins, as in the reference's second pass;
2. PROLONG from the first block one level coarser whose array holds the
   whole 6-point footprint of every point of the box, else from the first
   whose array holds the points' coincident or left coarse node (the taps
   past its edge are clamped, the reference's edge padding);
3. otherwise nothing: those ghosts keep their values (the outer boundary of
   the coarsest level, frozen at the initial data).

Boxes of one level are disjoint and read only interiors of that level or
arrays of the level below, so one launch per level runs them all. The
restriction plan (optional, applied after a step, finest level first)
injects each coarse interior node that coincides with a fine interior node,
first fine block in pool order winning.

Boxes are 6-tuples (x0, y0, z0, x1, y1, z1), half-open, in level units.
"""

from __future__ import annotations

import ctypes
from typing import Dict, List, Optional, Sequence, Tuple

import numpy as np

COPY, RESTRICT, PROLONG = 0, 1, 2

Box = Tuple[int, int, int, int, int, int]


class FillOp(ctypes.Structure):
    """Mirror of ``bssn_b200_fill_op`` in include/bssn_b200.h."""
    _fields_ = [("dst_off", ctypes.c_longlong), ("src_off", ctypes.c_longlong),
                ("point0", ctypes.c_longlong),
                ("dst_s", ctypes.c_int * 3), ("src_s", ctypes.c_int * 3),
                ("lo", ctypes.c_int * 3), ("hi", ctypes.c_int * 3),
                ("shift", ctypes.c_int * 3), ("kind", ctypes.c_int)]


def lagrange_weights(offsets: Sequence[int], target: float) -> np.ndarray:
    """Weights of the Lagrange polynomial through integer ``offsets``
    evaluated at ``target`` (kernels.py:36-46): w_j = prod_{m != j}
    (target - x_m) / (x_j - x_m), multiplied in offset order (the order
    fixes the last bit of each weight)."""
    w = []
    for j, xj in enumerate(offsets):
        p = 1.0
        for m, xm in enumerate(offsets):
            if m != j:
                p *= (target - xm) / (xj - xm)
        w.append(p)
    return np.array(w, dtype=np.float64)


MID_OFFSETS = (-2, -1, 0, 1, 2, 3)
W_MID = lagrange_weights(MID_OFFSETS, 0.5)


# ---------------------------------------------------------------- box algebra
def intersect(a: Box, b: Box) -> Optional[Box]:
    x0 = a[0] if a[0] > b[0] else b[0]
    x1 = a[3] if a[3] < b[3] else b[3]
    if x0 >= x1:
        return None
    y0 = a[1] if a[1] > b[1] else b[1]
    y1 = a[4] if a[4] < b[4] else b[4]
    if y0 >= y1:
        return None
    z0 = a[2] if a[2] > b[2] else b[2]
    z1 = a[5] if a[5] < b[5] else b[5]
    if z0 >= z1:
        return None
    return (x0, y0, z0, x1, y1, z1)


def subtract(a: Box, c: Box) -> List[Box]:
    """Disjoint boxes covering a minus c, where c = intersect(a, c) is not
    None (at most six: slabs cut off below and above c on each axis)."""
    out = []
    lo = [a[0], a[1], a[2]]
    hi = [a[3], a[4], a[5]]
    for ax in range(3):
        if lo[ax] < c[ax]:
            h = hi.copy()
            h[ax] = c[ax]
            out.append((lo[0], lo[1], lo[2], h[0], h[1], h[2]))
            lo[ax] = c[ax]
        if c[3 + ax] < hi[ax]:
            l2 = lo.copy()
            l2[ax] = c[3 + ax]
            out.append((l2[0], l2[1], l2[2], hi[0], hi[1], hi[2]))
            hi[ax] = c[3 + ax]
    return out


def volume(b: Box) -> int:
    return (b[3] - b[0]) * (b[4] - b[1]) * (b[5] - b[2])


def _carve(remaining: List[Box], region: Box, hit: List[Box]) -> List[Box]:
    """Split ``remaining`` by ``region``: the parts inside go to ``hit``,
    the parts outside are returned."""
    nxt = []
    for piece in remaining:
        x = intersect(piece, region)
        if x is None:
            nxt.append(piece)
        else:
            hit.append(x)
            nxt += subtract(piece, x)
    return nxt


# ---------------------------------------------------------------- lattice
class _Lat:
    """A block on its level's lattice: array start ``a`` (level units),
    extents ``S``, ghost width ``ng``, interior cells ``n``."""

    def __init__(self, blk, offset: int):
        q = [o / blk.h for o in blk.origin]
        oi = [int(round(v)) for v in q]
        if any(abs(v - r) > 1e-9 * max(1.0, abs(v)) for v, r in zip(q, oi)):
            raise ValueError(f"block origin {blk.origin} is not on its level lattice (h = {blk.h})")
        self.level = blk.level
        self.ng = blk.ng
        self.n = blk.n
        self.S = tuple(blk.shape)
        self.a = tuple(o - blk.ng for o in oi)
        self.offset = int(offset)
        a, S, g, n = self.a, self.S, self.ng, self.n
        self.array: Box = (a[0], a[1], a[2], a[0] + S[0], a[1] + S[1], a[2] + S[2])
        self.interior: Box = (a[0] + g, a[1] + g, a[2] + g, a[0] + g + n, a[1] + g + n, a[2] + g + n)

    def slabs(self) -> List[Box]:
        """The ghost shell as six disjoint slabs (level coordinates)."""
        a0, a1, a2, e0, e1, e2 = self.array
        i0, i1, i2, j0, j1, j2 = self.interior
        return [(a0, a1, a2, i0, e1, e2), (j0, a1, a2, e0, e1, e2),
                (i0, a1, a2, j0, i1, e2), (i0, j1, a2, j0, e1, e2),
                (i0, i1, a2, j0, j1, i2), (i0, i1, j2, j0, j1, e2)]


def _op(kind, dst: _Lat, src: _Lat, box: Box, shift) -> FillOp:
    op = FillOp()
    op.kind = kind
    op.dst_off, op.src_off = dst.offset, src.offset
    for i in range(3):
        op.dst_s[i], op.src_s[i] = dst.S[i], src.S[i]
        op.lo[i] = box[i] - dst.a[i]
        op.hi[i] = box[3 + i] - dst.a[i]
        op.shift[i] = int(shift[i])
    return op


class GhostPlan:
    """Fill and restriction op lists of a :class:`~bssn3d_b200.amr.BlockPool`.

    ``fill_lists``: [(level, [FillOp])] in ascending level order;
    ``restrict_lists``: [(level, [FillOp])] from the finest level down (each
    injects level ``level`` into level ``level - 1``). ``counts`` reports the
    ghost points by source kind (copy / prolong / none).
    """

    def __init__(self, pool, restrict: bool = False):
        self.pool = pool
        self.lat = [_Lat(b, pool.offsets[i]) for i, b in enumerate(pool.blocks)]
        by_level: Dict[int, List[int]] = {}
        for i, L in enumerate(self.lat):
            by_level.setdefault(L.level, []).append(i)
        self.levels = sorted(by_level)
        self._int = np.array([L.interior for L in self.lat], dtype=np.int64).reshape(-1, 6)
        self._arr = np.array([L.array for L in self.lat], dtype=np.int64).reshape(-1, 6)
        self.counts = {"copy": 0, "prolong": 0, "none": 0}
        self.fill_lists = []
        for lvl in self.levels:
            ops = []
            same = np.asarray(by_level[lvl], dtype=np.int64)
            coarse = np.asarray(by_level.get(lvl - 1, []), dtype=np.int64)
            for i in by_level[lvl]:
                ops += self._block_ops(i, same, coarse)
            if ops:
                self.fill_lists.append((lvl, ops))
        self.restrict_lists = []
        if restrict:
            for lvl in reversed(self.levels):
                if lvl - 1 not in by_level:
                    continue
                fine = np.asarray(by_level[lvl], dtype=np.int64)
                ops = []
                for c in by_level[lvl - 1]:
                    ops += self._restrict_ops(c, fine)
                if ops:
                    self.restrict_lists.append((lvl, ops))

    @staticmethod
    def _overlapping(boxes: np.ndarray, idx: np.ndarray, box: Box, scale: int = 1) -> List[int]:
        """Members of ``idx`` whose box (times ``scale``) meets ``box``."""
        if len(idx) == 0:
            return []
        b = boxes[idx] * scale
        hit = ((b[:, 0] < box[3]) & (b[:, 3] > box[0]) & (b[:, 1] < box[4]) & (b[:, 4] > box[1]) &
               (b[:, 2] < box[5]) & (b[:, 5] > box[2]))
        return [int(j) for j in idx[hit]]

    def _block_ops(self, i: int, same: np.ndarray, coarse: np.ndarray) -> List[FillOp]:
        b = self.lat[i]
        ops = []
        remaining = b.slabs()
        for j in self._overlapping(self._int, same, b.array):
            if j == i or not remaining:
                continue
            c = self.lat[j]
            hit: List[Box] = []
            remaining = _carve(remaining, c.interior, hit)
            shift = [b.a[k] - c.a[k] for k in range(3)]
            for x in hit:
                ops.append(_op(COPY, b, c, x, shift))
                self.counts["copy"] += volume(x)
        parents = self._overlapping(self._arr, coarse, b.array, scale=2)
        for reach in (4, 0):  # whole 6-point footprint inside, then coincident node inside
            for j in parents:
                if not remaining:
                    break
                p = self.lat[j]
                lo = [2 * p.a[k] + reach for k in range(3)]
                hi = [2 * p.a[k] + 2 * p.S[k] - (6 if reach else 1) for k in range(3)]
                hit = []
                remaining = _carve(remaining, (lo[0], lo[1], lo[2], hi[0], hi[1], hi[2]), hit)
                shift = [b.a[k] - 2 * p.a[k] for k in range(3)]
                for x in hit:
                    ops.append(_op(PROLONG, b, p, x, shift))
                    self.counts["prolong"] += volume(x)
        self.counts["none"] += sum(volume(r) for r in remaining)
        return ops

    def _restrict_ops(self, ci: int, fine: np.ndarray) -> List[FillOp]:
        c = self.lat[ci]
        ops = []
        remaining = [c.interior]
        big = tuple(2 * v for v in c.interior)
        for j in self._overlapping(self._int, fine, big):
            if not remaining:
                break
            f = self.lat[j]
            l0, l1, l2, h0, h1, h2 = f.interior
            # coarse nodes I with 2I inside the fine interior
            img = (-(-l0 // 2), -(-l1 // 2), -(-l2 // 2), (h0 - 1) // 2 + 1, (h1 - 1) // 2 + 1, (h2 - 1) // 2 + 1)
            hit = []
            remaining = _carve(remaining, img, hit)
            shift = [2 * c.a[k] - f.a[k] for k in range(3)]
            for x in hit:
                ops.append(_op(RESTRICT, c, f, x, shift))
        return ops


class DevicePlan:
    """The op lists validated by the C library and uploaded: one
    (level, ops_device, nops, npoints) entry per launch."""

    def __init__(self, plan: GhostPlan, device):
        import torch
        from . import _lib
        lib = _lib.load()
        self.fill = []
        self.restrict = []
        for dst, lists in ((self.fill, plan.fill_lists), (self.restrict, plan.restrict_lists)):
            for lvl, ops in lists:
                arr = (FillOp * len(ops))(*ops)
                total = lib.bssn_b200_fill_plan(ctypes.addressof(arr), len(ops), int(plan.pool.size))
                if total < 0:
                    _lib.check(_lib.EINVAL)
                raw = bytes(memoryview(arr).cast("B"))
                dev = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(device)
                dst.append((lvl, dev, len(ops), int(total)))
        self.wmid = (ctypes.c_double * 6)(*W_MID)

    def run(self, which: str, pool_tensor, stream) -> None:
        """Enqueue the ``"fill"`` (coarse to fine) or ``"restrict"`` (fine to
        coarse) launches on ``pool_tensor``."""
        for lvl, _, _, _ in getattr(self, which):
            self.run_level(which, lvl, pool_tensor, stream)

    def run_level(self, which: str, level: int, pool_tensor, stream) -> None:
        """Enqueue the one launch of ``which`` for ``level`` (if it has ops)."""
        from . import _lib
        lib = _lib.load()
        for lvl, dev, nops, npts in getattr(self, which):
            if lvl == level:
                _lib.check(lib.bssn_b200_fill(stream, pool_tensor.data_ptr(), dev.data_ptr(), nops, npts,
                                              ctypes.cast(self.wmid, ctypes.c_void_p)))
