"""The allocation-free constraint-norm entry point.

Some callers of this library cannot call cudaMalloc: an XLA FFI handler works
only with the buffers XLA passes in, a plugin inside a host application's CUDA
stream capture would break the capture by allocating, and some real-time loops
forbid allocation outright. ``bssn_b200_constraint_norms_static`` serves them:
it keeps its per-CTA partial sums in a static device array inside the library
instead of a caller-provided scratch buffer. This test calls it through the C
ABI twice in a row, on two different states, and checks both results against
the scratch-buffer entry point ``bssn_b200_constraint_norms``, to the 1e-12
relative tolerance of the other parity tests. The file is named to be collected last.
"""

import ctypes

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def test_static_norms_match_scratch_norms_twice():
    from bssn3d_b200 import _lib
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.fused_rhs import device_scalars, pack_S
    lib = _lib.load()
    dev = torch.device("cuda:0")
    grid, U, _ = ID.workload(0, n=24)
    Ud = torch.from_numpy(U).to(dev)
    S = device_scalars(pack_S(2.0, 0.0, 1.0, grid.dx, 0.0, 1.0, 0.0, (1, 1, 1, 1), (1, 0),
                              grid.dy, grid.dz), dev)
    _, Sx, Sy, Sz = Ud.shape
    stream = torch.cuda.current_stream(dev).cuda_stream

    need = int(lib.bssn_b200_norms_scratch_bytes())
    scratch = torch.empty(max(need // 8, 2), dtype=torch.float64, device=dev)

    def with_scratch(F):
        ref = torch.empty(2, dtype=torch.float64, device=dev)
        _lib.check(lib.bssn_b200_constraint_norms(stream, F.data_ptr(), S.data_ptr(), Sx, Sy, Sz,
                                                  grid.ng, scratch.data_ptr(), scratch.numel() * 8,
                                                  ref.data_ptr()))
        return ref.cpu().numpy()

    # the second call sees a different state, so a call that left stale
    # partial sums of the first one in the shared array would show
    Vd = Ud.clone()
    Vd[12:18] += 1e-2   # a traceful A~ changes both the Hamiltonian and momentum norms
    for F in (Ud, Vd):
        expect = with_scratch(F)
        assert np.all(np.isfinite(expect)) and expect[0] > 0
        out = torch.full((2,), np.nan, dtype=torch.float64, device=dev)
        _lib.check(lib.bssn_b200_constraint_norms_static(stream, F.data_ptr(), S.data_ptr(),
                                                         Sx, Sy, Sz, grid.ng, out.data_ptr()))
        got = out.cpu().numpy()
        np.testing.assert_allclose(got, expect, rtol=1e-12, atol=0)
    assert not np.allclose(with_scratch(Ud), with_scratch(Vd), rtol=1e-6)


def test_static_norms_reject_an_empty_interior():
    from bssn3d_b200 import _lib
    lib = _lib.load()
    F = torch.zeros((24, 6, 6, 6), dtype=torch.float64, device="cuda:0")
    S = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    out = torch.zeros(2, dtype=torch.float64, device="cuda:0")
    rc = lib.bssn_b200_constraint_norms_static(None, F.data_ptr(), S.data_ptr(), 6, 6, 6, 3, out.data_ptr())
    assert rc == _lib.EINVAL
    assert "interior" in lib.bssn_b200_last_error().decode()
