"""Halo staging of the stream kernel by bulk-tensor (TMA) copies
(BSSN_B200_STAGING=tma).

With the knob set, a state whose z extent is even and whose base is 16-byte
aligned is staged by one bulk-tensor copy per field and tile (edge tiles are
then clamped in shared memory); a state placed 8 bytes off a 16-byte boundary
cannot be, so it takes the default per-thread cp.async staging. Both paths
must give the same bytes for every kernel mode, and no bounded copy wait may
give up."""

import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

SHAPE = (18, 22, 64)   # interior and edge tiles on every axis


@pytest.fixture(autouse=True)
def _bulk_copy_staging(monkeypatch):
    monkeypatch.setenv("BSSN_B200_STAGING", "tma")


def _lib():
    from bssn3d_b200 import _lib as L
    return L, L.load()


def _state(seed=5, amp=0.05):
    rng = np.random.default_rng(seed)
    F = amp * rng.standard_normal((24,) + SHAPE)
    for k in (0, 1, 3, 6, 8):
        F[k] += 1.0
    return F


def _S(dt=0.02, t=0.4):
    from bssn3d_b200.fused_rhs import pack_S
    return pack_S(2.0, 0.06, dt, 0.1, 0.6, 20.0, t, (1, 1, 1, 1), (1, 0), 0.11, 0.09)


def _placed(a: np.ndarray, aligned: bool) -> torch.Tensor:
    """A device copy of ``a`` starting on a 16-byte boundary, or 8 bytes past one."""
    n = a.size
    base = torch.empty(n + 2, dtype=torch.float64, device="cuda")
    off = 0 if aligned else 1
    t = base[off:off + n].view(a.shape)
    t.copy_(torch.from_numpy(a))
    assert (t.data_ptr() % 16 == 0) == aligned
    return t


def _run(kind, aligned, ko_order=6, stage=1):
    L, lib = _lib()
    F = _state()
    U = _state(seed=6)
    A = _state(seed=7, amp=0.01)
    Fd, Ud, Ad = _placed(F, aligned), _placed(U, aligned), _placed(A, aligned)
    S = torch.from_numpy(_S()).cuda()
    Sx, Sy, Sz = SHAPE
    stream = torch.cuda.current_stream().cuda_stream
    if kind == "rhs":
        out = torch.empty_like(Fd)
        L.check(lib.bssn_b200_rhs(stream, Fd.data_ptr(), S.data_ptr(), out.data_ptr(), Sx, Sy, Sz))
        return out.cpu().numpy()
    if kind == "constraints":
        out = torch.empty((4,) + SHAPE, dtype=torch.float64, device="cuda")
        L.check(lib.bssn_b200_constraints(stream, Fd.data_ptr(), S.data_ptr(), out.data_ptr(), Sx, Sy, Sz))
        return out.cpu().numpy()
    if kind == "stage":
        nxt = _placed(np.zeros_like(F), aligned)
        L.check(lib.bssn_b200_rk4_stage(stream, stage, Ud.data_ptr(), Fd.data_ptr(), Ad.data_ptr(),
                                        nxt.data_ptr(), S.data_ptr(), 0.1, ko_order, 1e-4, 1e-4, Sx, Sy, Sz))
        return np.concatenate([nxt.cpu().numpy().ravel(), Ad.cpu().numpy().ravel()])
    if kind == "norms":
        need = int(lib.bssn_b200_norms_scratch_bytes())
        scratch = torch.empty(need // 8 + 1, dtype=torch.float64, device="cuda")
        out = torch.empty(2, dtype=torch.float64, device="cuda")
        L.check(lib.bssn_b200_constraint_norms(stream, Fd.data_ptr(), S.data_ptr(), Sx, Sy, Sz, 3,
                                               scratch.data_ptr(), need, out.data_ptr()))
        return out.cpu().numpy()
    raise ValueError(kind)


@pytest.mark.parametrize("kind,ko_order,stage", [("rhs", 6, 0), ("constraints", 6, 0), ("norms", 6, 0),
                                                 ("stage", 6, 1), ("stage", 6, 3), ("stage", 8, 2)])
def test_bulk_copies_and_per_thread_staging_agree_bitwise(kind, ko_order, stage):
    a = _run(kind, True, ko_order, stage)
    b = _run(kind, False, ko_order, stage)
    assert np.isfinite(a).all()
    np.testing.assert_array_equal(a, b)


def test_rhs_with_bulk_copies_vs_oracle():
    F = _state()
    got = _run("rhs", True)
    assert O.normwise_rel(got, O.rhs(F, _S())).max() < 1e-12


def test_no_bounded_copy_wait_gave_up():
    L, lib = _lib()
    count = ctypes.c_int(-1)
    L.check(lib.bssn_b200_async_copy_errors(ctypes.addressof(count)))
    assert count.value == 0
