"""Ozaki INT8 derivative path: the 138 derivatives (+ KO) of a state through
exact INT8 tensor-core contractions of k digit planes (include/bssn_b200.h,
``bssn_b200_ozaki_derivatives``), and the RHS built on them with the float64
algebra (``bssn_b200_rhs_algebra``): the algebra stays in float64, only the
stencils go through the tensor cores.

The reference has no Ozaki path for BSSN; its MCS Ozaki derivative
(2D/src/mcs2d/schemes/ozaki.py:257-380) is the design source.
"""

from __future__ import annotations

import torch

from . import _lib
from .fused_rhs import _stream_handle


class OzakiDerivatives:
    """Holds the device workspace for one grid shape and digit count."""

    def __init__(self, shape, k: int, device="cuda"):
        self.shape = tuple(int(s) for s in shape)
        self.k = int(k)
        self.device = torch.device(device)
        lib = _lib.load()
        need = int(lib.bssn_b200_ozaki_workspace_bytes(*self.shape, self.k))
        if need == 0:
            raise ValueError(f"bad Ozaki configuration shape={shape} k={k}")
        self.ws = torch.empty(need + 256, dtype=torch.uint8, device=self.device)
        off = (-self.ws.data_ptr()) % 256
        self.ptr = self.ws.data_ptr() + off
        self.bytes = need
        self.flag_ptr = lib.bssn_b200_ozaki_error_flag(self.ptr, *self.shape, self.k)

    def derivatives(self, Fs: torch.Tensor, S_dev: torch.Tensor, ko_sigma: float = 0.0,
                    ko_order: int = 6, out: torch.Tensor = None) -> torch.Tensor:
        lib = _lib.load()
        nslot = 138 + (24 if ko_sigma > 0 else 0)
        if out is None:
            out = torch.empty((nslot,) + self.shape, dtype=torch.float64, device=self.device)
        rc = lib.bssn_b200_ozaki_derivatives(_stream_handle(self.device), Fs.data_ptr(), S_dev.data_ptr(),
                                             out.data_ptr(), self.k, float(ko_sigma), int(ko_order),
                                             *self.shape, self.ptr, self.bytes)
        if rc != _lib.OK:
            raise _lib.BssnB200Error(rc, lib.bssn_b200_ozaki_last_error().decode())
        return out

    def check(self) -> None:
        """Raise if a tensor-core wait gave up (reads the flag in the workspace)."""
        off = int(self.flag_ptr) - self.ws.data_ptr()
        flag = self.ws[off:off + 4].view(torch.int32).item()
        if flag != 0:
            raise _lib.BssnB200Error(_lib.ECUDA, "Ozaki tensor-core wait gave up")

    def rhs(self, Fs: torch.Tensor, S_dev: torch.Tensor) -> torch.Tensor:
        """RHS with Ozaki derivatives and the float64 algebra (no KO)."""
        D = self.derivatives(Fs, S_dev)
        out = torch.empty_like(Fs)
        npts = Fs[0].numel()
        _lib.check(_lib.load().bssn_b200_rhs_algebra(_stream_handle(self.device), Fs.data_ptr(),
                                                      D.data_ptr(), S_dev.data_ptr(), out.data_ptr(), npts))
        return out
