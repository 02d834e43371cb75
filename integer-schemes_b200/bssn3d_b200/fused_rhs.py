"""The fused BSSN RHS entry point — drop-in for the reference's
``cuda_fused_algebra`` (3D/src/bssn3d/fused_rhs_cuda.py:62-72).

``cuda_fused_algebra(F, dx, dy, dz, eta, lmbda, lambda_f, cahd_c, dt, ssl_h,
ssl_sigma, t)`` takes the field dict keyed by ``FIELD_INPUTS`` and returns
``{field: d/dt}`` keyed by ``OUTPUT_FIELDS`` — the call ``BSSNSolver.rhs_dict``
makes for its fused schemes (3D/src/bssn3d/rhs.py:110-121). Fields are
float64 CUDA tensors (numpy arrays are accepted and copied to the current
device); the kernel is enqueued on torch's current stream.
"""

from __future__ import annotations

from typing import Mapping

import numpy as np
import torch

from . import _lib
from .state import FIELD_INPUTS, NUM_VARS, OUTPUT_FIELDS

NSCAL = 16
NOUT = len(OUTPUT_FIELDS)


def pack_S(eta, cahd_c, dt, dx, ssl_h, ssl_sigma, t, lmbda, lambda_f, dy, dz) -> np.ndarray:
    """The 16-scalar operand, in the order of fused_rhs_cuda.py:52-55."""
    return np.array([eta, cahd_c, dt, dx, ssl_h, ssl_sigma, t,
                     lmbda[0], lmbda[1], lmbda[2], lmbda[3], lambda_f[0], lambda_f[1],
                     dx, dy, dz], dtype=np.float64)


def scalars(p, dx, dy, dz, dt, t) -> np.ndarray:
    return pack_S(p.eta, p.cahd_c, dt, dx, p.ssl_h, p.ssl_sigma, t, p.lmbda, p.lambda_f, dy, dz)


def _stream_handle(device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def as_device_state(F, device=None) -> torch.Tensor:
    """Stack a field dict (or pass a (24, ...) array) into a contiguous CUDA tensor."""
    if isinstance(F, Mapping):
        arrs = [F[n] for n in FIELD_INPUTS]
        if isinstance(arrs[0], torch.Tensor):
            t = torch.stack(arrs)
        else:
            t = torch.from_numpy(np.stack([np.asarray(a, dtype=np.float64) for a in arrs]))
    elif isinstance(F, torch.Tensor):
        t = F
    else:
        t = torch.from_numpy(np.ascontiguousarray(F, dtype=np.float64))
    if t.dtype != torch.float64:
        raise TypeError(f"fields must be float64, got {t.dtype}")
    if not t.is_cuda:
        t = t.to(device or "cuda")
    if t.dim() != 4 or t.shape[0] != NUM_VARS:
        raise ValueError(f"fused: F must be (24, Sx, Sy, Sz), got {tuple(t.shape)}")
    return t.contiguous()


def device_scalars(S, device) -> torch.Tensor:
    S = torch.as_tensor(np.asarray(S, dtype=np.float64) if not isinstance(S, torch.Tensor) else S,
                        dtype=torch.float64)
    if S.numel() != NSCAL:
        raise ValueError(f"fused: S must have {NSCAL} scalars, got {S.numel()}")
    return S.to(device).contiguous()


def rhs_tensor(Fs: torch.Tensor, S_dev: torch.Tensor, out: torch.Tensor = None) -> torch.Tensor:
    """OUT (24, Sx, Sy, Sz) = RHS of the stacked state (one kernel launch)."""
    lib = _lib.load()
    if out is None:
        out = torch.empty_like(Fs)
    _, Sx, Sy, Sz = Fs.shape
    with torch.cuda.device(Fs.device):
        rc = lib.bssn_b200_rhs(_stream_handle(Fs.device), Fs.data_ptr(), S_dev.data_ptr(),
                               out.data_ptr(), Sx, Sy, Sz)
    _lib.check(rc)
    return out


def cuda_fused_algebra(F, dx, dy, dz, eta, lmbda, lambda_f, cahd_c, dt, ssl_h, ssl_sigma, t):
    """The fused scheme callable (fused_rhs_cuda.py:62-72 signature). Returns
    ``{field_name: d/dt}``; KO dissipation is not part of this call (it is the
    RK-stage entry's job, evolve.py:86-91)."""
    Fs = as_device_state(F)
    S = device_scalars(pack_S(eta, cahd_c, dt, dx, ssl_h, ssl_sigma, t, lmbda, lambda_f, dy, dz),
                       Fs.device)
    OUT = rhs_tensor(Fs, S)
    return {OUTPUT_FIELDS[k]: OUT[k] for k in range(NOUT)}


def device_rhs_fused(state, params, dx, dy, dz, dt, t=0.0):
    """``{field: d/dt}`` of a ``BSSNState`` (fused_rhs_cuda.py:75-80)."""
    p = params
    return cuda_fused_algebra(state.data, dx, dy, dz, p.eta, p.lmbda, p.lambda_f,
                              p.cahd_c, dt, p.ssl_h, p.ssl_sigma, t)


def derivatives(Fs: torch.Tensor, S_dev: torch.Tensor, ko_sigma: float = 0.0,
                ko_order: int = 6) -> torch.Tensor:
    """The 138 derivatives (+24 KO sums when ko_sigma > 0) of a stacked state."""
    lib = _lib.load()
    _, Sx, Sy, Sz = Fs.shape
    nslot = 138 + (24 if ko_sigma > 0 else 0)
    out = torch.empty((nslot, Sx, Sy, Sz), dtype=torch.float64, device=Fs.device)
    with torch.cuda.device(Fs.device):
        rc = lib.bssn_b200_derivatives(_stream_handle(Fs.device), Fs.data_ptr(), S_dev.data_ptr(),
                                       out.data_ptr(), float(ko_sigma), int(ko_order), Sx, Sy, Sz)
    _lib.check(rc)
    return out
