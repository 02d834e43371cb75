"""``BSSNSolver`` — the reference's RHS entry point (3D/src/bssn3d/rhs.py:63-139)
on the B200 fused kernel.

Same constructor and methods: ``rhs_dict(state, t, dt)`` returns
``{field: d/dt}`` over the full padded grid and ``rhs`` stacks it in
``VAR_NAMES`` order. ``dt`` defaults to ``0.25*dx`` (rhs.py:97-100). Only the
fused scheme exists here: ``"cuda_fused"`` (the reference's name for its
fused FFI scheme) and ``"cuda_b200"`` both select it; the reference's
XLA/Pallas schemes are not provided and raise ``ValueError``.
"""

from __future__ import annotations

from typing import Dict

from .fused_rhs import cuda_fused_algebra
from .grid import Grid, ghost_width
from .state import BSSNState, OUTPUT_FIELDS, PhysicsParams

SCHEMES = ("cuda_fused", "cuda_b200")


def _select_algebra(scheme: str):
    if scheme in SCHEMES:
        return cuda_fused_algebra
    raise ValueError(f"unknown scheme {scheme!r} (this build provides {SCHEMES})")


class BSSNSolver:
    def __init__(self, grid: Grid, params: PhysicsParams = None, order: int = 6,
                 dt: float = None, scheme: str = "cuda_b200", precision: str = "fp64",
                 ko_order: int = 8):
        self.grid = grid
        self.params = params or PhysicsParams()
        self.scheme = scheme
        if precision != "fp64":
            raise ValueError(f"unknown precision {precision!r} (fp64 only)")
        self.precision = precision
        if order != 6:
            raise ValueError(f"FD order {order} is not provided (order 6 only)")
        self.order = order
        self.ko_order = ko_order
        need = ghost_width(order, ko_order)
        if need > grid.ng:
            raise ValueError(
                f"FD order {order} / KO order {ko_order} need ng>={need} but grid has ng={grid.ng}.")
        self._algebra = _select_algebra(scheme)
        self.dt = dt if dt is not None else 0.25 * grid.dx

    def rhs_dict(self, state: BSSNState, t: float = 0.0, dt: float = None) -> Dict:
        g, p = self.grid, self.params
        data = state.data if isinstance(state, BSSNState) else state
        return self._algebra(data, g.dx, g.dy, g.dz, p.eta, p.lmbda, p.lambda_f,
                             p.cahd_c, self.dt if dt is None else dt, p.ssl_h, p.ssl_sigma, t)

    def rhs(self, state: BSSNState, t: float = 0.0, dt: float = None) -> BSSNState:
        import torch
        out = self.rhs_dict(state, t, dt)
        return BSSNState(torch.stack([out[name] for name in OUTPUT_FIELDS]))
