"""Slab split of one uniform block across ranks (one process per GPU).

The state (24, Sx, Sy, Sz) is cut along x, the outermost axis, into
contiguous ranges of planes, one per rank. A rank holds the planes it owns
plus ``halo`` planes on each side that its neighbours own (the stencil
reach: 3 for KO6, 4 for KO8), clipped to the array. Each RK stage is the
single-block stage kernel (``bssn_b200_rk4_stage``) over the whole local
array; then the halo planes of the stage's output are replaced by the
neighbours' owned planes: one ``batch_isend_irecv`` per stage with one
contiguous buffer per neighbour each way (NCCL between GPUs; the data lands
in this GPU's memory before the next launch reads it).

Why the owned planes come out exactly as in the single-block evolution:
every tap of an owned point lies inside the local array (its reach is at
most ``halo``), the only array ends where the kernel clamps its taps are the
global ends (rank 0's first plane, the last rank's last plane), and every
other operation of the stage is pointwise. The values the kernel writes at
halo planes come from clamped taps and are overwritten by the exchange
before anything reads them; they are the price of the split (2·halo extra
planes per interior rank). The plane ranges balance the planes each rank
evaluates, halos included.

Boundary condition: ``bc="none"`` (the Brill-Lindquist workloads). A
periodic x-axis would wrap through the first and last ranks and is not
provided for slabs.
"""

from __future__ import annotations

from typing import Callable, List, Optional, Tuple

import torch


def slab_ranges(Sx: int, world: int, halo: int) -> List[Tuple[int, int]]:
    """Owned plane ranges [a, b) per rank, contiguous and covering [0, Sx),
    balanced so that every rank evaluates about the same number of planes
    (owned + halo planes: ranks at the ends have one neighbour, the others
    two). Raises if a rank would own fewer than ``halo`` planes (its
    neighbours' halos would then reach past it)."""
    if world < 1:
        raise ValueError(f"world {world} < 1")
    nb = [(r > 0) + (r < world - 1) for r in range(world)]
    total = Sx + halo * sum(nb)
    base, extra = divmod(total, world)
    own = [base + (1 if r < extra else 0) - halo * nb[r] for r in range(world)]
    if world > 1 and min(own) < halo:
        raise ValueError(f"{Sx} planes over {world} ranks leaves a slab thinner than the "
                         f"{halo}-plane halo")
    out, a = [], 0
    for n in own:
        out.append((a, a + n))
        a += n
    assert a == Sx
    return out


class SlabLayout:
    """One rank's slab: owned planes [a, b) of the global array, local planes
    [la, lb) = [a - halo, b + halo) clipped to [0, Sx), and the halo
    transfers with its neighbours (global plane ranges)."""

    def __init__(self, Sx: int, world: int, rank: int, halo: int):
        if not 0 <= rank < world:
            raise ValueError(f"rank {rank} outside world {world}")
        self.Sx, self.world, self.rank, self.halo = int(Sx), int(world), int(rank), int(halo)
        self.ranges = slab_ranges(self.Sx, self.world, self.halo)
        self.a, self.b = self.ranges[rank]
        self.la = max(self.a - halo, 0)
        self.lb = min(self.b + halo, self.Sx)
        # (peer, global planes sent) and (peer, global planes received)
        self.sends, self.recvs = [], []
        if rank > 0:
            self.sends.append((rank - 1, (self.a, self.a + halo)))
            self.recvs.append((rank - 1, (self.la, self.a)))
        if rank < world - 1:
            self.sends.append((rank + 1, (self.b - halo, self.b)))
            self.recvs.append((rank + 1, (self.b, self.lb)))

    @property
    def local_planes(self) -> int:
        return self.lb - self.la

    def local_slice(self) -> slice:
        """The local planes as a slice of the global x axis."""
        return slice(self.la, self.lb)

    def owned_slice(self) -> slice:
        """The owned planes as a slice of the LOCAL x axis."""
        return slice(self.a - self.la, self.b - self.la)

    def to_local(self, planes: Tuple[int, int]) -> slice:
        return slice(planes[0] - self.la, planes[1] - self.la)

    def exchange_bytes(self, Sy: int, Sz: int) -> int:
        """Bytes this rank sends per exchange (24 float64 fields)."""
        return sum(8 * 24 * (hi - lo) * Sy * Sz for _, (lo, hi) in self.sends)


def exchange_halos(lay: SlabLayout, Y: torch.Tensor, group=None) -> None:
    """Replace the halo planes of the local array ``Y`` (24, lb-la, Sy, Sz)
    by the neighbours' owned planes: one packed buffer per neighbour each
    way, one ``batch_isend_irecv``."""
    if lay.world == 1:
        return
    import torch.distributed as dist
    ops, recv = [], []
    for q, planes in lay.sends:
        ops.append(dist.P2POp(dist.isend, Y[:, lay.to_local(planes)].contiguous(), q, group=group))
    for p, planes in lay.recvs:
        sl = lay.to_local(planes)
        buf = torch.empty_like(Y[:, sl])
        recv.append((sl, buf))
        ops.append(dist.P2POp(dist.irecv, buf, p, group=group))
    for req in dist.batch_isend_irecv(ops):
        req.wait()
    for sl, buf in recv:
        Y[:, sl].copy_(buf)


def exchange_halos_local(lays: List[SlabLayout], Ys: List[torch.Tensor]) -> None:
    """The same exchange between slabs held by one process (all ranks'
    local arrays in ``Ys``): plain copies from each owner's planes."""
    for lay, Y in zip(lays, Ys):
        for p, planes in lay.recvs:
            Y[:, lay.to_local(planes)].copy_(Ys[p][:, lays[p].to_local(planes)])


StageFn = Callable[[int, torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor, torch.Tensor], None]


class SlabEvolution:
    """RK4 on one uniform block split into x-slabs across ranks.

    ``stage_fn(stage, U, Y, ACC, YNEXT, S)`` runs one RK stage on a local
    array; the default is the fused stage kernel through
    ``BSSNEvolution`` (ghost width, KO and floors as given). The per-stage
    halo exchange uses ``torch.distributed`` point-to-point on ``group``.
    """

    def __init__(self, grid, params=None, world: int = 1, rank: int = 0, ko_sigma: float = 0.1,
                 ko_order: int = 6, bc: str = "none", group=None, stage_fn: Optional[StageFn] = None):
        if bc != "none":
            raise ValueError(f"bc {bc!r}: the slab split supports bc='none' only")
        from .evolve import BSSNEvolution
        self.grid = grid
        self.evo = BSSNEvolution(grid, params, ko_sigma=ko_sigma, bc="none", ko_order=ko_order)
        self.halo = max(3, int(ko_order) // 2)
        self.layout = SlabLayout(grid.shape[0], world, rank, self.halo)
        self.group = group
        self.stage_fn = stage_fn if stage_fn is not None else self.evo._stage

    def local(self, U_global: torch.Tensor) -> torch.Tensor:
        """This rank's local array (owned + halo planes) cut from a global state."""
        return U_global[:, self.layout.local_slice()].clone()

    def owned(self, U_local: torch.Tensor) -> torch.Tensor:
        return U_local[:, self.layout.owned_slice()]

    def scalars(self, t: float, dt: float, device) -> torch.Tensor:
        return self.evo._S(t, dt, device)

    def buffers(self, U: torch.Tensor):
        key = (tuple(U.shape), U.device)
        b = getattr(self, "_bufs", None)
        if b is None or b[0] != key:
            b = (key, {name: torch.empty_like(U) for name in ("Ya", "Yb", "ACC")})
            self._bufs = b
        return b[1]

    def step_inplace(self, U: torch.Tensor, S: torch.Tensor) -> None:
        b = self.buffers(U)
        for stage, (y, ynext) in enumerate([(U, b["Ya"]), (b["Ya"], b["Yb"]), (b["Yb"], b["Ya"]),
                                            (b["Ya"], U)]):
            self.stage_fn(stage, U, y, b["ACC"], ynext, S)
            exchange_halos(self.layout, ynext, self.group)

    def advance_time(self, S: torch.Tensor) -> None:
        if S.is_cuda:
            self.evo._advance_time(S)
        else:
            S[6] += S[2]

    def evolve(self, U_local: torch.Tensor, dt: float, nsteps: int, t0: float = 0.0) -> torch.Tensor:
        U = U_local.clone()
        S = self.scalars(t0, dt, U.device)
        for _ in range(int(nsteps)):
            self.step_inplace(U, S)
            self.advance_time(S)
        return U

    def gather(self, U_local: torch.Tensor) -> Optional[torch.Tensor]:
        """The global state assembled from every rank's owned planes
        (returned on every rank; one all-gather of padded slabs)."""
        lay = self.layout
        if lay.world == 1:
            return U_local.clone()
        import torch.distributed as dist
        width = max(b - a for a, b in lay.ranges)
        pad = torch.zeros((24, width) + tuple(U_local.shape[2:]), dtype=U_local.dtype,
                          device=U_local.device)
        own = self.owned(U_local)
        pad[:, :own.shape[1]].copy_(own)
        parts = [torch.empty_like(pad) for _ in range(lay.world)]
        dist.all_gather(parts, pad, group=self.group)
        return torch.cat([parts[r][:, :b - a] for r, (a, b) in enumerate(lay.ranges)], dim=1)

    @staticmethod
    def evolve_in_one_process(slabs: List["SlabEvolution"], U_locals: List[torch.Tensor], dt: float,
                              nsteps: int, t0: float = 0.0) -> List[torch.Tensor]:
        """Every rank's slab stepped by one process (one device): per stage,
        each slab's stage launch, then the halo copies between the slabs.
        The same schedule as the distributed run, without a process group."""
        lays = [s.layout for s in slabs]
        Us = [U.clone() for U in U_locals]
        Ss = [s.scalars(t0, dt, U.device) for s, U in zip(slabs, Us)]
        bufs = [s.buffers(U) for s, U in zip(slabs, Us)]
        for _ in range(int(nsteps)):
            for stage in range(4):
                outs = []
                for s, U, S, b in zip(slabs, Us, Ss, bufs):
                    y, ynext = [(U, b["Ya"]), (b["Ya"], b["Yb"]), (b["Yb"], b["Ya"]), (b["Ya"], U)][stage]
                    s.stage_fn(stage, U, y, b["ACC"], ynext, S)
                    outs.append(ynext)
                exchange_halos_local(lays, outs)
            for s, S in zip(slabs, Ss):
                s.advance_time(S)
        return Us

    def constraint_sums(self, U_local: torch.Tensor) -> torch.Tensor:
        """(sum H^2, sum |M|^2, count) over this rank's owned interior
        planes: the constraints of the local array (halos current), one
        launch of ``bssn_b200_constraints``, summed on the device."""
        from . import _lib
        from .fused_rhs import _stream_handle, device_scalars, pack_S
        lay, g = self.layout, self.grid
        ng = g.ng
        _, nx, Sy, Sz = U_local.shape
        S = device_scalars(pack_S(2.0, 0.0, 1.0, g.dx, 0.0, 1.0, 0.0, (1, 1, 1, 1), (1, 0),
                                  g.dy, g.dz), U_local.device)
        out = torch.empty((4, nx, Sy, Sz), dtype=torch.float64, device=U_local.device)
        with torch.cuda.device(U_local.device):
            _lib.check(_lib.load().bssn_b200_constraints(_stream_handle(U_local.device),
                                                         U_local.data_ptr(), S.data_ptr(),
                                                         out.data_ptr(), nx, Sy, Sz))
        lo, hi = max(lay.a, ng), min(lay.b, lay.Sx - ng)
        sums = torch.zeros(3, dtype=torch.float64, device=U_local.device)
        if hi > lo:
            C = out[:, lay.to_local((lo, hi)), ng:Sy - ng, ng:Sz - ng]
            sums[0] = (C[0] * C[0]).sum()
            sums[1] = (C[1] * C[1] + C[2] * C[2] + C[3] * C[3]).sum()
            sums[2] = float(C[0].numel())
        return sums

    def constraint_norms(self, U_local: torch.Tensor) -> Tuple[float, float]:
        """Interior norms (H, |M|) of the global state
        (3D/src/bssn3d/constraints.py:53-62): every rank's
        :meth:`constraint_sums`, one all-reduce of the three sums."""
        sums = self.constraint_sums(U_local)
        if self.layout.world > 1:
            import torch.distributed as dist
            dist.all_reduce(sums, group=self.group)
        hm = torch.sqrt(sums[:2] / sums[2])
        return float(hm[0]), float(hm[1])
