"""Batched AMR block lists for the BSSN RHS / RK4 stage.

The reference has no BSSN AMR (3D/src/mcs3d/amr/__init__.py:1); its block-
structured AMR exists for 2D MCS (2D/src/mcs2d/amr/state.py:77) and the 3D
multipatch scalar wave (3D/src/multipatch/amr/state.py). This module builds
what the batched workloads need: an uneven list of cubic blocks of mixed
sizes on nested refinement levels around the punctures, each with its own
ghost zones filled from the analytic Brill-Lindquist formula, stored back to
back in one pooled device buffer, plus the block table the batched kernels
walk (one persistent launch per RK stage over every block).

Ghosts, two ways (``BatchedEvolution(ghosts=...)``):

* ``"evolve"``: each block is evolved on its own, ghosts included, with the
  same clamped-stencil RHS as a single uniform block;
* ``"exchange"``: before every stage the ghosts are refilled from the other
  blocks (same-level copies, prolongation from the level below; the plan is
  built in :mod:`bssn3d_b200.ghosts`), and the stage kernels update the
  interiors only, like the reference's AMR step
  (3D/src/multipatch/amr/evolve.py:94-147). Ghosts with no source block keep
  their initial values (a frozen outer boundary).

Pool layout: block b occupies doubles [offset_b, offset_b + 24*n_b) with
n_b = Sx*Sy*Sz, field f of block b at offset_b + f*n_b, each field C order
(z contiguous) — the single-block layout, repeated.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass
from typing import List, Sequence, Tuple

import numpy as np

from .grid import Grid
from .initial_data import Puncture, brill_lindquist


class BlockDesc(ctypes.Structure):
    """Mirror of ``bssn_b200_block`` in include/bssn_b200.h."""
    _fields_ = [("offset", ctypes.c_longlong),
                ("sx", ctypes.c_int), ("sy", ctypes.c_int), ("sz", ctypes.c_int),
                ("tile0", ctypes.c_int),
                ("h", ctypes.c_double * 3),
                ("core", ctypes.c_int), ("reserved", ctypes.c_int)]


@dataclass(frozen=True)
class Block:
    level: int
    n: int                                 # interior cells per axis
    origin: Tuple[float, float, float]     # first interior node
    h: float                               # grid spacing of the level
    ng: int = 3

    @property
    def shape(self):
        s = self.n + 2 * self.ng
        return (s, s, s)

    @property
    def points(self) -> int:
        return int(np.prod(self.shape))

    @property
    def interior_points(self) -> int:
        return self.n ** 3

    def grid(self) -> Grid:
        return Grid(Nx=self.n, Ny=self.n, Nz=self.n, dx=self.h, dy=self.h, dz=self.h, ng=self.ng,
                    xmin=self.origin[0], ymin=self.origin[1], zmin=self.origin[2])


def nested_blocks(count: int, levels: int, punctures: Sequence[Puncture], domain: float,
                  coarse_h: float, seed: int, sizes=(16, 24, 32), probs=(0.5, 0.3, 0.2),
                  ng: int = 3) -> List[Block]:
    """``count`` blocks on ``levels`` refinement levels (factor 2).

    Level l has spacing coarse_h / 2^l and covers a box of half-width
    domain / 2^(l+1) around a puncture (the heavier one twice as often);
    block interiors are drawn from ``sizes`` with ``probs`` and their origins
    snapped to the level's lattice, all from ``numpy.random.default_rng(seed)``.
    Level populations grow with l (finer levels need more, smaller blocks).
    """
    rng = np.random.default_rng(seed)
    w = np.array([2.0 ** l for l in range(levels)])
    lvl_p = w / w.sum()
    masses = np.array([p.mass for p in punctures])
    punct_p = masses ** 0.5 / (masses ** 0.5).sum()
    blocks = []
    for _ in range(count):
        lvl = int(rng.choice(levels, p=lvl_p))
        n = int(rng.choice(sizes, p=probs))
        pc = punctures[int(rng.choice(len(punctures), p=punct_p))].position
        h = coarse_h / 2 ** lvl
        half = domain / 2 ** (lvl + 1)
        centre = np.array(pc) + rng.uniform(-half, half, 3)
        origin = np.round((centre - 0.5 * n * h) / h) * h
        blocks.append(Block(level=lvl, n=n, origin=tuple(float(o) for o in origin), h=h, ng=ng))
    return blocks


def workload(index: int, count: int = None, ng: int = 3):
    """(blocks, punctures, dt) of the numbered batched workload.

    3: 600 blocks, 3 levels, q = 1/10 (m1 = 0.909 at x = -0.5, m2 = 0.0909 at x = +5),
       domain [-8,8]^3, coarse h = 0.25
    4: 2000 blocks, 5 levels, q = 1/100 (m1 = 0.990 at 0, m2 = 0.0099 at x = 6),
       domain [-32,32]^3, coarse h = 1.0
    dt = 0.25 x the finest spacing present (one global step for every block).
    """
    if index == 3:
        punct = [Puncture(0.909, (-0.5, 0.0, 0.0)), Puncture(0.0909, (5.0, 0.0, 0.0))]
        blocks = nested_blocks(600 if count is None else count, 3, punct, 16.0, 0.25,
                               seed=20261203 + 3, ng=ng)
    elif index == 4:
        punct = [Puncture(0.990, (0.0, 0.0, 0.0)), Puncture(0.0099, (6.0, 0.0, 0.0))]
        blocks = nested_blocks(2000 if count is None else count, 5, punct, 64.0, 1.0,
                               seed=20261203 + 4, ng=ng)
    else:
        raise ValueError(f"unknown batched workload {index}")
    dt = 0.25 * min(b.h for b in blocks)
    return blocks, punct, dt


class BlockPool:
    """Host-side layout of a block list: offsets, total size, descriptor table."""

    def __init__(self, blocks: Sequence[Block], tile=(4, 4, 16)):
        self.blocks = list(blocks)
        self.offsets = np.zeros(len(self.blocks), dtype=np.int64)
        off = 0
        for i, b in enumerate(self.blocks):
            self.offsets[i] = off
            off += 24 * b.points
        self.size = off                    # doubles per pooled state
        self.tile = tuple(tile)
        self.table, self.ntiles = self.descriptors(self.tile)

    def descriptors(self, tile, core: bool = False, active=None):
        """Block table and tile count; ``core=True`` leaves each block's ghost
        layers out of the tiles (they come from a ghost fill); ``active``
        (block indices) limits the table to the blocks a launch evolves."""
        TX, TY, TZ = tile
        idx = list(range(len(self.blocks))) if active is None else list(active)
        arr = (BlockDesc * len(idx))()
        t0 = 0
        for j, i in enumerate(idx):
            b = self.blocks[i]
            sx, sy, sz = b.shape
            d = arr[j]
            d.offset = int(self.offsets[i])
            d.sx, d.sy, d.sz = sx, sy, sz
            d.tile0 = t0
            d.h[0] = d.h[1] = d.h[2] = b.h
            d.core = b.ng if core else 0
            c2 = 2 * d.core
            t0 += -(-(sx - c2) // TX) * -(-(sy - c2) // TY) * -(-(sz - c2) // TZ)
        return arr, t0

    @property
    def interior_points(self) -> int:
        return sum(b.interior_points for b in self.blocks)

    @property
    def points(self) -> int:
        return sum(b.points for b in self.blocks)

    def gather(self, pooled: np.ndarray, i: int) -> np.ndarray:
        b = self.blocks[i]
        o = int(self.offsets[i])
        return pooled[o:o + 24 * b.points].reshape((24,) + b.shape)

    def scatter(self, pooled: np.ndarray, i: int, data: np.ndarray) -> None:
        b = self.blocks[i]
        o = int(self.offsets[i])
        pooled[o:o + 24 * b.points] = data.reshape(-1)

    def initial_state(self, punctures, seed: int = 0) -> np.ndarray:
        """Brill-Lindquist data on every block (ghosts included), pooled."""
        out = np.empty(self.size)
        for i, b in enumerate(self.blocks):
            self.scatter(out, i, brill_lindquist(b.grid(), punctures, noise_sigma=1e-8, seed=seed + i))
        return out


# ---------------------------------------------------------------------------
# device side
# ---------------------------------------------------------------------------

class BatchedEvolution:
    """RK4 over a pooled block list: each stage is ONE persistent launch of
    ``bssn_b200_batch_rk4_stage`` covering every block, and ``evolve`` replays
    the captured step (4 stage launches + the time advance) as a CUDA graph.

    ``variant`` picks the kernel's tile shape (include/bssn_b200.h); use
    :func:`autotune` to choose it for a given block list.
    """

    ORDERS = ("pool", "size")

    def __init__(self, pool: BlockPool, params=None, ko_sigma: float = 0.1, ko_order: int = 6,
                 variant: int = 0, device="cuda", ghosts: str = "evolve", restrict: bool = False,
                 plan=None, active=None, order: str = "pool"):
        import torch
        from .state import PhysicsParams
        from . import _lib
        if ghosts not in ("evolve", "exchange"):
            raise ValueError(f"ghosts must be 'evolve' or 'exchange', not {ghosts!r}")
        if restrict and ghosts != "exchange":
            raise ValueError("restrict needs ghosts='exchange'")
        self.ghosts = ghosts
        self.pool = pool
        # blocks the stage kernels evolve (all, unless a rank holds mirrors of remote blocks)
        self.active = list(range(len(pool.blocks))) if active is None else list(active)
        self.params = params or PhysicsParams()
        self.ko_sigma = float(ko_sigma)
        self.ko_order = int(ko_order)
        ng_need = max(3, ko_order // 2)
        if any(b.ng < ng_need for b in pool.blocks):
            raise ValueError(f"KO order {ko_order} needs ng >= {ng_need} on every block")
        self.device = torch.device(device)
        self._lib = _lib
        self.plan = None
        self.dplan = None
        if ghosts == "exchange":
            from .ghosts import DevicePlan, GhostPlan
            self.plan = plan if plan is not None else GhostPlan(pool, restrict=restrict)
            self.dplan = DevicePlan(self.plan, self.device)
        self.order = "pool"
        self.set_variant(variant, order)
        self._bufs = None

    def launch_order(self, order: str):
        """The active blocks in the order their tiles are laid out for the
        persistent launch (the block-to-CTA mapping: CTA c takes global tiles
        c, c + grid, ...): ``"pool"`` keeps pool order; ``"size"`` puts the
        largest blocks first, so the last tiles handed out are small ones."""
        if order == "pool":
            return list(self.active)
        if order == "size":
            return sorted(self.active, key=lambda i: (-self.pool.blocks[i].points, i))
        raise ValueError(f"order must be one of {self.ORDERS}, not {order!r}")

    def set_variant(self, variant: int, order: str = None) -> None:
        """Tile variant and block order of the batched stage launches."""
        import torch
        lib = self._lib.load()
        order = self.order if order is None else order
        table, _ = self.pool.descriptors(self.pool.tile, core=self.ghosts == "exchange",
                                         active=self.launch_order(order))
        ntiles = lib.bssn_b200_batch_plan(ctypes.addressof(table), len(self.active), int(variant))
        if ntiles < 0:
            self._lib.check(self._lib.EINVAL)
        raw = bytes(memoryview(table).cast("B"))
        self.table_dev = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(self.device)
        self.ntiles = int(ntiles)
        self.variant = int(variant)
        self.order = order

    def scalars(self, t: float, dt: float):
        from .fused_rhs import device_scalars, scalars
        h = self.pool.blocks[0].h
        return device_scalars(scalars(self.params, h, h, h, dt, t), self.device)

    def _stream(self):
        import torch
        return torch.cuda.current_stream(self.device).cuda_stream

    def buffers(self, U):
        import torch
        if self._bufs is None or self._bufs["Ya"].shape != U.shape:
            self._bufs = {k: torch.empty_like(U) for k in ("Ya", "Yb", "ACC")}
            if self.ghosts == "exchange":
                self.seed_buffers(U)
        return self._bufs

    def seed_buffers(self, U):
        """With ghost exchange the stage kernels write interiors only, so the
        stage buffers' unfilled ghosts (the frozen outer boundary) must hold
        U's values: copy U into them."""
        b = self.buffers(U)
        b["Ya"].copy_(U)
        b["Yb"].copy_(U)

    def fill(self, Y):
        """Refill the ghosts of the pooled state Y, coarse level first."""
        if self.dplan is not None:
            self.dplan.run("fill", Y, self._stream())

    def restrict(self, U):
        """Inject fine interiors into the coarser levels, finest first."""
        if self.dplan is not None:
            self.dplan.run("restrict", U, self._stream())

    def stage(self, stage, U, Y, ACC, YNEXT, S):
        p = self.params
        lib = self._lib.load()
        rc = lib.bssn_b200_batch_rk4_stage(self._stream(), stage, U.data_ptr(), Y.data_ptr(), ACC.data_ptr(),
                                           YNEXT.data_ptr(), S.data_ptr(), self.ko_sigma, self.ko_order,
                                           p.chi_floor, p.alpha_floor, self.table_dev.data_ptr(),
                                           len(self.active), self.ntiles, self.variant)
        self._lib.check(rc)

    def rhs(self, U, S):
        """Pooled RHS (no KO), the batched ``cuda_fused_algebra``. With ghost
        exchange the ghosts of a copy of U are filled first and only the
        interiors of the result are written (the rest is zero)."""
        import torch
        if self.ghosts == "exchange":
            U = U.clone()
            self.fill(U)
            out = torch.zeros_like(U)
        else:
            out = torch.empty_like(U)
        rc = self._lib.load().bssn_b200_batch_rhs(self._stream(), U.data_ptr(), S.data_ptr(), out.data_ptr(),
                                                  self.table_dev.data_ptr(), len(self.active),
                                                  self.ntiles, self.variant)
        self._lib.check(rc)
        return out

    def step_inplace(self, U, S):
        b = self.buffers(U)
        for stage, (y, ynext) in enumerate([(U, b["Ya"]), (b["Ya"], b["Yb"]), (b["Yb"], b["Ya"]),
                                            (b["Ya"], U)]):
            self.fill(y)
            self.stage(stage, U, y, b["ACC"], ynext, S)
        if self.plan is not None and self.plan.restrict_lists:
            self.restrict(U)

    def advance_time(self, S):
        self._lib.check(self._lib.load().bssn_b200_advance_time(self._stream(), S.data_ptr()))

    def capture(self, U, S):
        """One captured step (4 batched stage launches + time advance) on
        static copies of U and S; replay advances them by one step."""
        import torch
        U_g, S_g = U.clone(), S.clone()
        self.buffers(U_g)
        if self.ghosts == "exchange":
            self.seed_buffers(U_g)
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            pu, ps = U_g.clone(), S_g.clone()
            self.step_inplace(pu, ps)
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        del pu, ps
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.step_inplace(U_g, S_g)
            self.advance_time(S_g)
        # a graph does not own the memory it replays on: keep its static
        # tensors, stage buffers and plan tables alive with the graph object
        g.static_tensors = (U_g, S_g, self.buffers(U_g), self.table_dev, self.dplan)
        return g, U_g, S_g

    def evolve(self, U, dt: float, nsteps: int, t0: float = 0.0):
        S = self.scalars(t0, dt)
        g, U_g, _ = self.capture(U, S)
        for _ in range(int(nsteps)):
            g.replay()
        return U_g

    # -- the comparison point: one launch per block per stage ----------------
    def per_block_tables(self):
        """One single-block table per active block (same kernel, same tile
        variant, same covered points as the persistent launch), in one device
        buffer: (buffer, byte offsets, tile counts)."""
        import torch
        lib = self._lib.load()
        table, _ = self.pool.descriptors(self.pool.tile, core=self.ghosts == "exchange", active=self.active)
        raw, offs, ntiles = bytearray(), [], []
        for j in range(len(self.active)):
            one = BlockDesc.from_buffer_copy(table[j])
            n = lib.bssn_b200_batch_plan(ctypes.addressof(one), 1, self.variant)
            if n < 0:
                self._lib.check(self._lib.EINVAL)
            offs.append(len(raw))
            ntiles.append(int(n))
            raw += bytes(memoryview(one).cast("B"))
            raw += bytes((-len(raw)) % 16)
        return torch.frombuffer(raw, dtype=torch.uint8).to(self.device), offs, ntiles

    def per_block_launch_step_inplace(self, U, S, tables=None):
        """The RK4 step of :meth:`step_inplace` with one batched-stage launch
        per block (a one-entry block table each) instead of one persistent
        launch over all blocks: the same kernel, tiles and results, so the
        difference in time is the launch structure alone."""
        lib = self._lib.load()
        buf, offs, ntiles = tables if tables is not None else self.per_block_tables()
        b = self.buffers(U)
        p = self.params
        for stage, (y, ynext) in enumerate([(U, b["Ya"]), (b["Ya"], b["Yb"]), (b["Yb"], b["Ya"]),
                                            (b["Ya"], U)]):
            self.fill(y)
            for o, nt in zip(offs, ntiles):
                rc = lib.bssn_b200_batch_rk4_stage(self._stream(), stage, U.data_ptr(), y.data_ptr(),
                                                   b["ACC"].data_ptr(), ynext.data_ptr(), S.data_ptr(),
                                                   self.ko_sigma, self.ko_order, p.chi_floor, p.alpha_floor,
                                                   buf.data_ptr() + o, 1, nt, self.variant)
                self._lib.check(rc)
        if self.plan is not None and self.plan.restrict_lists:
            self.restrict(U)

    def capture_per_block(self, U, S):
        """:meth:`capture` for the one-launch-per-block step."""
        import torch
        tables = self.per_block_tables()
        U_g, S_g = U.clone(), S.clone()
        self.buffers(U_g)
        if self.ghosts == "exchange":
            self.seed_buffers(U_g)
        side = torch.cuda.Stream(self.device)
        side.wait_stream(torch.cuda.current_stream(self.device))
        with torch.cuda.stream(side):
            pu, ps = U_g.clone(), S_g.clone()
            self.per_block_launch_step_inplace(pu, ps, tables)
        torch.cuda.current_stream(self.device).wait_stream(side)
        torch.cuda.synchronize(self.device)
        del pu, ps
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.per_block_launch_step_inplace(U_g, S_g, tables)
            self.advance_time(S_g)
        g.static_tensors = (U_g, S_g, self.buffers(U_g), tables[0], self.dplan)
        return g, U_g, S_g

    def per_block_step_inplace(self, U, S_blocks):
        """The same RK4 step with one uniform-kernel launch per block per
        stage (``S_blocks[i]`` carries block i's spacing); blocks evolve on
        their own, so this compares with ``ghosts="evolve"`` only."""
        if self.ghosts != "evolve":
            raise ValueError("per-block launches evolve ghosts themselves: use ghosts='evolve'")
        lib = self._lib.load()
        b = self.buffers(U)
        p = self.params
        for stage, (y, ynext) in enumerate([("U", "Ya"), ("Ya", "Yb"), ("Yb", "Ya"), ("Ya", "U")]):
            for i, blk in enumerate(self.pool.blocks):
                o = int(self.pool.offsets[i])
                m = 24 * blk.points
                views = {k: (U if k == "U" else b[k])[o:o + m] for k in ("U", "Ya", "Yb", "ACC")}
                sx, sy, sz = blk.shape
                rc = lib.bssn_b200_rk4_stage(self._stream(), stage, views["U"].data_ptr(), views[y].data_ptr(),
                                             views["ACC"].data_ptr(), views[ynext].data_ptr(),
                                             S_blocks[i].data_ptr(), self.ko_sigma, self.ko_order,
                                             p.chi_floor, p.alpha_floor, sx, sy, sz)
                self._lib.check(rc)

    def constraint_sums(self, U, filled: bool = False):
        """Device tensor (sum of H^2, sum of |M|^2, point count) over the
        interior points of the blocks this object evolves: each block's norms
        come from the fused norm kernel (constraints.py:53-62 per block) and
        are weighted by its interior point count. With ghost exchange the
        ghosts of a copy of U are filled first (unless ``filled``)."""
        import torch
        from .fused_rhs import device_scalars, pack_S
        lib = self._lib.load()
        if self.ghosts == "exchange" and not filled:
            U = U.clone()
            self.fill(U)
        need = int(lib.bssn_b200_norms_scratch_bytes())
        scratch = torch.empty(need // 8 + 1, dtype=torch.float64, device=self.device)
        out = torch.empty(len(self.active), 2, dtype=torch.float64, device=self.device)
        for j, i in enumerate(self.active):
            blk = self.pool.blocks[i]
            S = device_scalars(pack_S(2.0, 0.0, 1.0, blk.h, 0.0, 1.0, 0.0, (1, 1, 1, 1), (1, 0),
                                      blk.h, blk.h), self.device)
            o = int(self.pool.offsets[i])
            sx, sy, sz = blk.shape
            rc = lib.bssn_b200_constraint_norms(self._stream(), U[o:].data_ptr(), S.data_ptr(), sx, sy, sz,
                                                blk.ng, scratch.data_ptr(), need, out[j].data_ptr())
            self._lib.check(rc)
        w = torch.tensor([float(self.pool.blocks[i].interior_points) for i in self.active], dtype=torch.float64,
                         device=self.device)
        return torch.cat([(out ** 2 * w[:, None]).sum(0), w.sum().reshape(1)])

    def constraint_norms(self, U):
        """Interior L2 norms (H, |M|) over every block's interior points together."""
        import torch
        sums = self.constraint_sums(U)
        hm = torch.sqrt(sums[:2] / sums[2])
        return float(hm[0]), float(hm[1])

    def block_scalars(self, t: float, dt: float):
        from .fused_rhs import device_scalars, scalars
        return [device_scalars(scalars(self.params, blk.h, blk.h, blk.h, dt, t), self.device)
                for blk in self.pool.blocks]


def autotune(evo: BatchedEvolution, U, dt: float, variants=None, orders=None, reps: int = 3):
    """Time one captured RK4 step for every (tile variant, block order) on
    this block list and keep the fastest. The tile shape and the block-to-CTA
    mapping are the kernel's launch knobs; its register cap is fixed at one
    255-register CTA per SM (a two-CTA, 128-register build of the same kernel
    spills ~3.7 KB per thread and measured slower on B200). Returns
    {(variant, order): ms} and leaves ``evo`` on the winner."""
    import torch
    from . import _lib
    variants = range(_lib.NVARIANTS) if variants is None else variants
    orders = BatchedEvolution.ORDERS if orders is None else orders
    times = {}
    for v in variants:
        for order in orders:
            evo.set_variant(v, order)
            g, U_g, _ = evo.capture(U, evo.scalars(0.0, dt))
            g.replay()
            torch.cuda.synchronize(evo.device)
            best = float("inf")
            for _ in range(reps):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                g.replay()
                b.record()
                b.synchronize()
                best = min(best, a.elapsed_time(b))
            times[(v, order)] = best
            del g, U_g
    v, order = min(times, key=times.get)
    evo.set_variant(v, order)
    return times
