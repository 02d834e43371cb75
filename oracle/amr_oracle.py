"""TEST INFRASTRUCTURE — CPU oracle of the AMR ghost fill and restriction.

Only tests/ import this module, and only as the checker of the CUDA fill
kernel (``bssn_b200_fill``) and of the batched exchange step.

It restates the reference's node-centred transfer operators
(3D/src/multipatch/amr/kernels.py) with numpy and decides every ghost
point's source point by point from the block geometry, without the box
planner of the package:

* ``refine_axis`` / ``refine``: 2:1 node-centred refinement of a WHOLE block
  along one axis / x then y then z, the parent edge-padded by (2, 3)
  (kernels.py:52-71; prolongate, :76-102, refines the full parent and
  crops);
* ``fill``: for each level from coarse to fine and each block, every ghost
  point takes (1) the first other same-level block, in pool order, whose
  interior holds it (exact copy, sync.py:105-122), else (2) the value of the
  refined array of the first block one level coarser whose array holds the
  point's whole 6-point footprint, else of the first whose array holds its
  coincident or left node (sync.py:70-88 with the reference's edge padding),
  else (3) keeps its value;
* ``restrict``: finest level first, each coarse interior node that
  coincides with a fine interior node takes that node's value, first fine
  block in pool order (injection, kernels.py:114-145).

Block geometry comes as ``(level, a, S, ng, offset)`` with ``a`` the array
start on the level's node lattice (so the interior is [a+ng, a+S-ng)).
"""

from __future__ import annotations

from typing import Dict, List, Sequence

import numpy as np

OFFSETS = (-2, -1, 0, 1, 2, 3)


def midpoint_weights() -> np.ndarray:
    """Lagrange weights at +1/2 for OFFSETS (kernels.py:36-49), in the same
    multiplication order."""
    w = []
    for j, xj in enumerate(OFFSETS):
        p = 1.0
        for m, xm in enumerate(OFFSETS):
            if m != j:
                p *= (0.5 - xm) / (xj - xm)
        w.append(p)
    return np.array(w)


W = midpoint_weights()


def refine_axis(c: np.ndarray, axis: int) -> np.ndarray:
    """fine[2k] = c[k], fine[2k+1] = sum_j W[j] c[clamp(k + OFFSETS[j])],
    summed from 0 in offset order (kernels.py:52-71)."""
    N = c.shape[axis]
    pad = [(0, 0)] * c.ndim
    pad[axis] = (2, 3)
    P = np.pad(c, pad, mode="edge")
    mids = 0.0
    for w, off in zip(W, OFFSETS):
        sl = [slice(None)] * c.ndim
        sl[axis] = slice(2 + off, 2 + off + N)
        mids = mids + w * P[tuple(sl)]
    shape = list(c.shape)
    shape[axis] = 2 * N
    out = np.empty(shape)
    ev = [slice(None)] * c.ndim
    od = [slice(None)] * c.ndim
    ev[axis] = slice(0, 2 * N, 2)
    od[axis] = slice(1, 2 * N, 2)
    out[tuple(ev)] = c
    out[tuple(od)] = mids
    return out


def refine(block: np.ndarray) -> np.ndarray:
    """(24, S) -> (24, 2S): x, then y, then z (kernels.py:96-98)."""
    r = block
    for ax in (1, 2, 3):
        r = refine_axis(r, ax)
    return r


class Geometry:
    def __init__(self, level: int, a, S, ng: int, offset: int):
        self.level = int(level)
        self.a = np.array(a, dtype=np.int64)
        self.S = np.array(S, dtype=np.int64)
        self.ng = int(ng)
        self.offset = int(offset)

    def view(self, pool: np.ndarray) -> np.ndarray:
        n = int(np.prod(self.S))
        return pool[self.offset:self.offset + 24 * n].reshape((24,) + tuple(int(s) for s in self.S))

    def interior_holds(self, g: np.ndarray) -> np.ndarray:
        lo = self.a + self.ng
        hi = self.a + self.S - self.ng
        return np.all((g >= lo) & (g < hi), axis=1)


def _ghost_points(G: Geometry) -> np.ndarray:
    """Local indices (m, 3) of the block's ghost points."""
    S = [int(s) for s in G.S]
    idx = np.indices(S).reshape(3, -1).T
    inner = np.all((idx >= G.ng) & (idx < np.array(S) - G.ng), axis=1)
    return idx[~inner]


def sources(geo: Sequence[Geometry], b: int):
    """Per ghost point of block b: (local index, kind, source block) with kind
    0 copy, 2 prolong, -1 none."""
    G = geo[b]
    loc = _ghost_points(G)
    glob = loc + G.a
    kind = np.full(len(loc), -1)
    src = np.full(len(loc), -1)
    for j, C in enumerate(geo):
        if j == b or C.level != G.level:
            continue
        m = (kind < 0) & C.interior_holds(glob)
        kind[m], src[m] = 0, j
    for reach in ("safe", "contain"):
        for j, P in enumerate(geo):
            if P.level != G.level - 1:
                continue
            g = glob - 2 * P.a
            if reach == "safe":
                ok = np.all((g >= 4) & (g <= 2 * P.S - 7), axis=1)
            else:
                ok = np.all((g >= 0) & (g <= 2 * P.S - 2), axis=1)
            m = (kind < 0) & ok
            kind[m], src[m] = 2, j
    return loc, kind, src


def fill(pool: np.ndarray, geo: Sequence[Geometry], blocks: Sequence[int] = None) -> np.ndarray:
    """The filled pool (a copy). ``blocks`` limits the destinations checked
    (their sources are always the full pool filled coarse-first)."""
    out = pool.copy()
    levels = sorted({G.level for G in geo})
    refined: Dict[int, np.ndarray] = {}
    for lvl in levels:
        for b, G in enumerate(geo):
            if G.level != lvl:
                continue
            if blocks is not None and b not in blocks and not any(
                    geo[d].level > lvl for d in blocks):
                continue
            loc, kind, src = sources(geo, b)
            dst = G.view(out)
            for j in np.unique(src[kind >= 0]):
                m = src == j
                Sg = geo[j]
                if kind[m][0] == 0:
                    sl = loc[m] + G.a - Sg.a
                    dst[:, loc[m, 0], loc[m, 1], loc[m, 2]] = Sg.view(out)[:, sl[:, 0], sl[:, 1], sl[:, 2]]
                else:
                    if j not in refined:
                        refined[j] = refine(Sg.view(out))
                    g = loc[m] + G.a - 2 * Sg.a
                    dst[:, loc[m, 0], loc[m, 1], loc[m, 2]] = refined[j][:, g[:, 0], g[:, 1], g[:, 2]]
        refined.clear()  # the next level prolongs from this one, now complete
    return out


def restrict(pool: np.ndarray, geo: Sequence[Geometry]) -> np.ndarray:
    out = pool.copy()
    levels = sorted({G.level for G in geo}, reverse=True)
    for lvl in levels:
        for c, C in enumerate(geo):
            if C.level != lvl - 1:
                continue
            S = [int(s) for s in C.S]
            idx = np.indices(S).reshape(3, -1).T
            idx = idx[np.all((idx >= C.ng) & (idx < np.array(S) - C.ng), axis=1)]
            glob2 = 2 * (idx + C.a)
            done = np.zeros(len(idx), bool)
            dst = C.view(out)
            for f, Fg in enumerate(geo):
                if Fg.level != lvl:
                    continue
                m = ~done & Fg.interior_holds(glob2)
                if m.any():
                    s = glob2[m] - Fg.a
                    dst[:, idx[m, 0], idx[m, 1], idx[m, 2]] = Fg.view(out)[:, s[:, 0], s[:, 1], s[:, 2]]
                    done |= m
    return out


def geometry_of(pool) -> List[Geometry]:
    """Geometry of a package BlockPool (origins on the level lattice)."""
    out = []
    for i, b in enumerate(pool.blocks):
        a = [int(round(o / b.h)) - b.ng for o in b.origin]
        out.append(Geometry(b.level, a, b.shape, b.ng, pool.offsets[i]))
    return out
