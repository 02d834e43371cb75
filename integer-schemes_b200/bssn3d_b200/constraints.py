"""``ConstraintSolver`` — Hamiltonian and momentum constraints on the GPU
(3D/src/bssn3d/constraints.py:38-62).

``constraints(state)`` returns ``{'H', 'M0', 'M1', 'M2'}`` over the padded
grid (one fused launch: 6th-order derivatives + constraint algebra);
``l2(state)`` returns the interior norms (RMS of H and
sqrt(mean(M0^2 + M1^2 + M2^2)) over ``[ng:-ng]^3``).
"""

from __future__ import annotations

from typing import Dict, Tuple

import torch

from . import _lib
from .fused_rhs import _stream_handle, as_device_state, device_scalars, pack_S
from .grid import Grid
from .state import BSSNState


class ConstraintSolver:
    def __init__(self, grid: Grid, order: int = 6):
        if order != 6:
            raise ValueError(f"order {order} is not provided (order 6 only)")
        if grid.ng < 3:
            raise ValueError(f"order {order} needs ng>=3, grid ng={grid.ng}")
        self.grid = grid
        self._partials = {}

    def constraints_tensor(self, state) -> torch.Tensor:
        U = as_device_state(state.data if isinstance(state, BSSNState) else state)
        g = self.grid
        S = device_scalars(pack_S(2.0, 0.0, 1.0, g.dx, 0.0, 1.0, 0.0, (1, 1, 1, 1), (1, 0),
                                  g.dy, g.dz), U.device)
        out = torch.empty((4,) + tuple(U.shape[1:]), dtype=torch.float64, device=U.device)
        _, Sx, Sy, Sz = U.shape
        with torch.cuda.device(U.device):
            rc = _lib.load().bssn_b200_constraints(_stream_handle(U.device), U.data_ptr(),
                                                   S.data_ptr(), out.data_ptr(), Sx, Sy, Sz)
        _lib.check(rc)
        return out

    def constraints(self, state) -> Dict[str, torch.Tensor]:
        out = self.constraints_tensor(state)
        return {"H": out[0], "M0": out[1], "M1": out[2], "M2": out[3]}

    def l2_tensor(self, state) -> torch.Tensor:
        """(H_l2, M_l2) as a 2-element device tensor: one fused launch plus a
        fixed-order reduction of its per-CTA partial sums."""
        U = as_device_state(state.data if isinstance(state, BSSNState) else state)
        g = self.grid
        S = device_scalars(pack_S(2.0, 0.0, 1.0, g.dx, 0.0, 1.0, 0.0, (1, 1, 1, 1), (1, 0),
                                  g.dy, g.dz), U.device)
        lib = _lib.load()
        out = torch.empty(2, dtype=torch.float64, device=U.device)
        _, Sx, Sy, Sz = U.shape
        with torch.cuda.device(U.device):
            need = int(lib.bssn_b200_norms_scratch_bytes())
            key = U.device.index
            buf = self._partials.get(key)
            if buf is None or buf.numel() * 8 < need:
                buf = torch.empty(max(need // 8, 2), dtype=torch.float64, device=U.device)
                self._partials[key] = buf
            rc = lib.bssn_b200_constraint_norms(_stream_handle(U.device), U.data_ptr(), S.data_ptr(),
                                                Sx, Sy, Sz, g.ng, buf.data_ptr(), buf.numel() * 8,
                                                out.data_ptr())
        _lib.check(rc)
        return out

    def l2(self, state) -> Tuple[float, float]:
        """Interior norms (H, |M|) as Python floats (one device-to-host read)."""
        h, m = self.l2_tensor(state).tolist()
        return h, m
