"""24-field BSSN state and gauge parameters.

Mirrors the reference's ``BSSNState`` / ``PhysicsParams``
(3D/src/bssn3d/state.py:26-155): the same field order, the same upper-
triangular symmetric-tensor index map and the same parameter defaults. The
state is a ``(24, Sx, Sy, Sz)`` float64 torch tensor, normally resident on a
CUDA device.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Tuple

import torch

ALPHA = 0
CHI = 1
K = 2
GT0, GT1, GT2, GT3, GT4, GT5 = 3, 4, 5, 6, 7, 8
BETA0, BETA1, BETA2 = 9, 10, 11
AT0, AT1, AT2, AT3, AT4, AT5 = 12, 13, 14, 15, 16, 17
GTILDE0, GTILDE1, GTILDE2 = 18, 19, 20
B0, B1, B2 = 21, 22, 23
NUM_VARS = 24

VAR_NAMES = [
    "alpha", "chi", "K",
    "gt0", "gt1", "gt2", "gt3", "gt4", "gt5",
    "beta0", "beta1", "beta2",
    "At0", "At1", "At2", "At3", "At4", "At5",
    "Gt0", "Gt1", "Gt2",
    "B0", "B1", "B2",
]
NAME_TO_IDX = {name: i for i, name in enumerate(VAR_NAMES)}
# the fused entry point's input and output orders are the state order
FIELD_INPUTS = list(VAR_NAMES)
OUTPUT_FIELDS = list(VAR_NAMES)

SYM_IDX = {
    (0, 0): 0, (0, 1): 1, (0, 2): 2, (1, 1): 3, (1, 2): 4, (2, 2): 5,
    (1, 0): 1, (2, 0): 2, (2, 1): 4,
}


class BSSNState:
    """24-field BSSN state as one ``(24, Sx, Sy, Sz)`` float64 tensor."""

    def __init__(self, data: torch.Tensor):
        if data.dim() != 4 or data.shape[0] != NUM_VARS:
            raise ValueError(f"state must be (24, Sx, Sy, Sz), got {tuple(data.shape)}")
        self.data = data

    @property
    def alpha(self): return self.data[ALPHA]
    @property
    def chi(self): return self.data[CHI]
    @property
    def K(self): return self.data[K]
    @property
    def beta(self): return self.data[BETA0:BETA0 + 3]
    @property
    def Gt(self): return self.data[GTILDE0:GTILDE0 + 3]
    @property
    def B(self): return self.data[B0:B0 + 3]
    @property
    def gt(self): return self.data[GT0:GT0 + 6]
    @property
    def At(self): return self.data[AT0:AT0 + 6]

    def gt_ij(self, i: int, j: int): return self.data[GT0 + SYM_IDX[(i, j)]]
    def At_ij(self, i: int, j: int): return self.data[AT0 + SYM_IDX[(i, j)]]

    @property
    def shape(self): return tuple(self.data.shape[1:])

    @classmethod
    def minkowski(cls, shape: Tuple[int, int, int], device="cuda") -> "BSSNState":
        data = torch.zeros((NUM_VARS,) + tuple(shape), dtype=torch.float64, device=device)
        for k in (ALPHA, CHI, GT0, GT3, GT5):
            data[k] = 1.0
        return cls(data)


@dataclass(frozen=True)
class PhysicsParams:
    """Gauge / damping parameters (3D/src/bssn3d/state.py:113-155 defaults)."""

    eta: float = 2.0
    lmbda: Tuple[float, float, float, float] = (1.0, 1.0, 1.0, 1.0)
    lambda_f: Tuple[float, float] = (1.0, 0.0)
    cahd_c: float = 0.06
    ssl_h: float = 0.6
    ssl_sigma: float = 20.0
    chi_floor: float = 1.0e-4
    alpha_floor: float = 1.0e-4
    alpha_inf: float = 1.0
    chi_inf: float = 1.0

    def lam(self, i: int) -> float:
        return self.lmbda[i]
