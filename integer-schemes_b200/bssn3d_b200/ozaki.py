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
from .amr import BatchedEvolution
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


NKIND = 5  # pass kinds of one derivative bundle (bssn_b200_batch_ozaki_plan)


def ozaki_plan(table, nblocks: int):
    """Host plan of a block table for the batched Ozaki calls: (tile0 as a
    flat list of 5 * nblocks first tiles, the 5 per-kind tile totals as a
    ctypes array, pts0 as a list, covered point total)."""
    import ctypes
    lib = _lib.load()
    tile0 = (ctypes.c_int * (NKIND * nblocks))()
    ntiles = (ctypes.c_longlong * NKIND)()
    pts0 = (ctypes.c_longlong * nblocks)()
    npts = lib.bssn_b200_batch_ozaki_plan(ctypes.addressof(table), nblocks, tile0, ntiles, pts0)
    if npts < 0:
        raise _lib.BssnB200Error(_lib.EINVAL, lib.bssn_b200_ozaki_last_error().decode())
    return list(tile0), ntiles, list(pts0), int(npts)


class BatchedOzakiEvolution(BatchedEvolution):
    """RK4 over a pooled block list with the Ozaki INT8 derivative path. Each
    stage is the ghost fill (``ghosts="exchange"``), ONE derivative bundle of
    every block (``bssn_b200_batch_ozaki_derivatives``: the 138 derivatives
    and 24 KO sums into a pooled slot buffer, k digit planes per value) and
    ONE stage update from those derivatives (``bssn_b200_batch_rk4_stage_derivs``:
    the float64 algebra and the RK4 update at the covered points). The
    FP64 path it is measured against is :class:`BatchedEvolution` on the same
    pool; everything else (fills, restriction, norms, capture) is shared.
    """

    def __init__(self, pool, k: int, params=None, ko_sigma: float = 0.1, ko_order: int = 6,
                 device="cuda", ghosts: str = "exchange", restrict: bool = False, plan=None, active=None):
        super().__init__(pool, params=params, ko_sigma=ko_sigma, ko_order=ko_order, variant=0,
                         device=device, ghosts=ghosts, restrict=restrict, plan=plan, active=active)
        if not 1 <= int(k) <= 8:
            raise ValueError(f"k must be 1..8, not {k}")
        self.k = int(k)
        table, _ = pool.descriptors(pool.tile, core=ghosts == "exchange", active=self.active)
        n = len(self.active)
        tile0, self.ntiles_kind, pts0, self.npoints = ozaki_plan(table, n)
        raw = bytes(memoryview(table).cast("B"))
        self.oz_table = torch.frombuffer(bytearray(raw), dtype=torch.uint8).to(self.device)
        self.tile0_dev = torch.tensor(tile0, dtype=torch.int32, device=self.device)
        self.pts0_dev = torch.tensor(pts0, dtype=torch.int64, device=self.device)
        self.nslot = 162 if self.ko_sigma > 0 else 138
        self.D = torch.empty(pool.size // 24 * self.nslot, dtype=torch.float64, device=self.device)
        self.ws = torch.zeros(512, dtype=torch.uint8, device=self.device)
        self.ws_ptr = self.ws.data_ptr() + (-self.ws.data_ptr()) % 256

    def derivatives(self, Y, S):
        """The derivative bundle of every block of Y into ``self.D``."""
        lib = _lib.load()
        rc = lib.bssn_b200_batch_ozaki_derivatives(self._stream(), Y.data_ptr(), S.data_ptr(), self.D.data_ptr(),
                                                   self.k, self.ko_sigma, self.ko_order, self.oz_table.data_ptr(),
                                                   len(self.active), self.tile0_dev.data_ptr(), self.ntiles_kind,
                                                   self.ws_ptr, 256)
        if rc != _lib.OK:
            raise _lib.BssnB200Error(rc, lib.bssn_b200_ozaki_last_error().decode())
        return self.D

    def derivative_view(self, i: int):
        """Block i's (nslot, sx, sy, sz) view of the derivative pool."""
        b = self.pool.blocks[i]
        o = int(self.pool.offsets[i]) // 24 * self.nslot
        return self.D[o:o + self.nslot * b.points].view((self.nslot,) + tuple(b.shape))

    def stage(self, stage, U, Y, ACC, YNEXT, S):
        self.derivatives(Y, S)
        p = self.params
        rc = _lib.load().bssn_b200_batch_rk4_stage_derivs(
            self._stream(), stage, U.data_ptr(), Y.data_ptr(), ACC.data_ptr(), YNEXT.data_ptr(), self.D.data_ptr(),
            S.data_ptr(), int(self.ko_sigma > 0), p.chi_floor, p.alpha_floor, self.oz_table.data_ptr(),
            len(self.active), self.pts0_dev.data_ptr(), self.npoints)
        _lib.check(rc)

    def check(self) -> None:
        """Raise if a tensor-core wait gave up in any launch so far."""
        off = self.ws_ptr - self.ws.data_ptr()
        if self.ws[off:off + 4].view(torch.int32).item() != 0:
            raise _lib.BssnB200Error(_lib.ECUDA, "Ozaki tensor-core wait gave up")

    def rhs(self, U, S):
        raise NotImplementedError("the Ozaki block-list path advances states; use BatchedEvolution.rhs")

    def capture(self, U, S):
        g, U_g, S_g = super().capture(U, S)
        g.static_tensors = g.static_tensors + (self.D, self.ws, self.oz_table, self.tile0_dev, self.pts0_dev,
                                               self.ntiles_kind)
        return g, U_g, S_g


def interior_field_errors(pool, A, B):
    """Per field, over the interiors of every block of the pooled arrays:
    max |A - B| / max |B| (0 where both vanish)."""
    import torch
    num = torch.zeros(24, dtype=torch.float64, device=A.device)
    den = torch.zeros(24, dtype=torch.float64, device=A.device)
    for i, b in enumerate(pool.blocks):
        o = int(pool.offsets[i])
        g = b.ng
        a = A[o:o + 24 * b.points].view((24,) + tuple(b.shape))[:, g:-g, g:-g, g:-g]
        r = B[o:o + 24 * b.points].view((24,) + tuple(b.shape))[:, g:-g, g:-g, g:-g]
        num = torch.maximum(num, (a - r).abs().amax(dim=(1, 2, 3)))
        den = torch.maximum(den, r.abs().amax(dim=(1, 2, 3)))
    err = torch.where(num == 0, torch.zeros_like(num), num / den.clamp_min(1e-300))
    return [float(x) for x in err.cpu()]


def choose_k(pool, U, dt: float, ks=(5, 6, 7, 8), bar: float = 1e-10, ghosts: str = "exchange",
             ko_sigma: float = 0.0, ko_order: int = 6, device="cuda"):
    """The autotuner's digit-count knob: the smallest k in ``ks`` whose RHS
    on this block list and state U (the first RK4 stage's accumulator, with
    KO only if ``ko_sigma`` > 0) stays within ``bar`` of the float64 block
    path for every field: max |oz - fp64| / max |fp64| over the interiors,
    the per-field measure of the 192^3 sweep. Without KO, fields whose RHS
    vanishes identically (shift and gauge fields of time-symmetric data)
    match exactly; with KO their rates are float64 rounding noise of near-unit
    values and the per-field ratio loses its meaning.
    Returns (k or None, {k: worst field error})."""
    import torch
    fp = BatchedEvolution(pool, ko_sigma=ko_sigma, ko_order=ko_order, device=device, ghosts=ghosts)
    Y = U.clone()
    fp.fill(Y)
    S = fp.scalars(0.0, dt)
    ref, tmp = torch.zeros_like(U), torch.empty_like(U)
    fp.stage(0, Y, Y, ref, tmp, S)
    plan = fp.plan
    del fp
    errs, chosen = {}, None
    for k in ks:
        oz = BatchedOzakiEvolution(pool, k=k, ko_sigma=ko_sigma, ko_order=ko_order, device=device,
                                   ghosts=ghosts, plan=plan)
        acc = torch.zeros_like(U)
        oz.stage(0, Y, Y, acc, tmp, S)
        oz.check()
        errs[k] = max(interior_field_errors(pool, acc, ref))
        del oz, acc
        torch.cuda.empty_cache()
        if chosen is None and errs[k] <= bar:
            chosen = k
    return chosen, errs
