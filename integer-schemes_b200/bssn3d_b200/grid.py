"""Vertex-centred, ghost-padded uniform grid (3D/src/bssn3d/grid.py:14-50).

Nodes are ``x_k = xmin + k*dx`` for ``k = -ng .. Nx+ng-1`` with
``dx = (hi - lo) / N``. The ghost width is the widest stencil's reach,
``max(order, ko_order) // 2`` (common/src/mcs_common/derivatives.py:51-76).
"""

from __future__ import annotations

from dataclasses import dataclass

import numpy as np

FD_ORDERS = (6,)
KO_ORDERS = (6, 8)


def ghost_width(order: int = 6, ko_order: int = 8) -> int:
    if order not in (4, 6, 8) or ko_order not in (4, 6, 8):
        raise ValueError(f"unsupported FD order {order} / KO order {ko_order}")
    return max(order, ko_order) // 2


@dataclass
class Grid:
    Nx: int
    Ny: int
    Nz: int
    dx: float
    dy: float
    dz: float
    ng: int
    xmin: float = -0.5
    ymin: float = -0.5
    zmin: float = -0.5

    def __post_init__(self):
        ng = self.ng
        self.x = self.xmin + np.arange(-ng, self.Nx + ng) * self.dx
        self.y = self.ymin + np.arange(-ng, self.Ny + ng) * self.dy
        self.z = self.zmin + np.arange(-ng, self.Nz + ng) * self.dz

    @property
    def shape(self):
        return (self.Nx + 2 * self.ng, self.Ny + 2 * self.ng, self.Nz + 2 * self.ng)

    @property
    def interior_points(self) -> int:
        return self.Nx * self.Ny * self.Nz

    def mesh(self):
        return np.meshgrid(self.x, self.y, self.z, indexing="ij")

    @classmethod
    def from_domain(cls, N, order=6, lo=-0.5, hi=0.5, ko_order=8, ng=None):
        """Cubic domain ``[lo, hi]^3`` with ``N`` interior cells per axis."""
        if isinstance(N, int):
            N = (N, N, N)
        g = ghost_width(order, ko_order) if ng is None else int(ng)
        d = [(hi - lo) / n for n in N]
        return cls(Nx=N[0], Ny=N[1], Nz=N[2], dx=d[0], dy=d[1], dz=d[2],
                   ng=g, xmin=lo, ymin=lo, zmin=lo)
