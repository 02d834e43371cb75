"""Ozaki INT8 derivative path (tcgen05, kind::i8) against the float64 oracle:
error falls with the digit count k, k = 8 reproduces float64 to rounding,
repeated runs are bit-identical, and the RHS built on the INT8 derivatives
with the float64 algebra meets 1e-10 per field at k >= 6 on Brill-Lindquist
data."""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _state(n=16, seed=0):
    from bssn3d_b200 import initial_data as ID
    grid, U, dt = ID.workload(1, n=n)
    return grid, U, dt


def _S(grid, dt):
    from bssn3d_b200.fused_rhs import pack_S
    return pack_S(2.0, 0.06, dt, grid.dx, 0.6, 20.0, 0.0, (1, 1, 1, 1), (1, 0), grid.dy, grid.dz)


def _slot_scales(U, h):
    """Natural error scale of every derivative slot: max|f| / h^p of its field
    (p = 1 for first, 2 for second derivatives). The digit split is exact to
    2^-7k of a line's largest value, so errors are measured against the field,
    not against the derivative (the diagonal metric of Brill-Lindquist data is
    1 to within 1e-16 and its derivatives are rounding noise)."""
    from bssn3d_b200.state import VAR_NAMES
    fmax = np.abs(U.reshape(24, -1)).max(axis=1)
    g2 = [0, 1, 3, 4, 5, 6, 7, 8, 9, 10, 11]
    sc = np.empty(138)
    for f in range(24):
        sc[3 * f:3 * f + 3] = fmax[f] / h
    for m, f in enumerate(g2):
        sc[72 + 6 * m:72 + 6 * m + 6] = fmax[f] / h ** 2
    return np.maximum(sc, 1e-300), fmax


def test_ozaki_derivatives_converge_with_k_and_repeat():
    from bssn3d_b200.ozaki import OzakiDerivatives
    from bssn3d_b200.fused_rhs import device_scalars
    grid, U, dt = _state(n=20)
    S = _S(grid, dt)
    Ud = torch.from_numpy(U).cuda()
    Sd = device_scalars(S, "cuda")
    ref = O.derivatives(U, grid.dx, grid.dy, grid.dz)
    ko = O.ko(U, grid.dx, grid.dy, grid.dz, 0.1, 6)
    sc, fmax = _slot_scales(U, grid.dx)
    ko_sc = np.maximum(0.1 * fmax / grid.dx, 1e-300)
    errs = []
    for k in (5, 6, 7, 8):
        oz = OzakiDerivatives(U.shape[1:], k)
        D = oz.derivatives(Ud, Sd, ko_sigma=0.1, ko_order=6)
        oz.check()
        Dn = D.cpu().numpy()
        e = (np.abs(Dn[:138] - ref).reshape(138, -1).max(axis=1) / sc).max()
        ek = (np.abs(Dn[138:] - ko).reshape(24, -1).max(axis=1) / ko_sc).max()
        errs.append(max(e, ek))
        if k == 8:
            for _ in range(4):
                np.testing.assert_array_equal(oz.derivatives(Ud, Sd, ko_sigma=0.1, ko_order=6).cpu().numpy(), Dn)
    assert errs[0] < 1e-8
    assert errs[-1] < 1e-13
    assert errs[1] < errs[0] and errs[2] < errs[1]


def test_ozaki_rhs_meets_1e10_per_field():
    from bssn3d_b200.ozaki import OzakiDerivatives
    from bssn3d_b200.fused_rhs import device_scalars
    grid, U, dt = _state(n=24)
    S = _S(grid, dt)
    ref = O.rhs(U, S)
    Ud = torch.from_numpy(U).cuda()
    for k in (6, 7, 8):
        oz = OzakiDerivatives(U.shape[1:], k)
        out = oz.rhs(Ud, device_scalars(S, "cuda")).cpu().numpy()
        oz.check()
        err = O.normwise_rel(out, ref)
        assert err.max() <= 1e-10, (k, err.max(), int(np.argmax(err)))


def test_ozaki_rejects_bad_arguments():
    from bssn3d_b200 import _lib
    lib = _lib.load()
    F = torch.zeros((24, 10, 10, 10), dtype=torch.float64, device="cuda")
    assert lib.bssn_b200_ozaki_workspace_bytes(10, 10, 10, 9) == 0
    ws = torch.empty(1 << 20, dtype=torch.uint8, device="cuda")
    rc = lib.bssn_b200_ozaki_derivatives(None, F.data_ptr(), F.data_ptr(), F.data_ptr(), 9, 0.0, 6,
                                         10, 10, 10, ws.data_ptr(), 1 << 20)
    assert rc == _lib.EINVAL
    assert "k must be" in lib.bssn_b200_ozaki_last_error().decode()


@pytest.mark.parametrize("k,ko_order", [(5, 6), (6, 8), (8, 6)])
def test_ozaki_bundle_equals_cpu_restatement_bit_for_bit(k, ko_order):
    """Every slot of the tensor-core bundle equals the numpy restatement of the
    same digit split, integer contraction and recombination order."""
    from bssn3d_b200.fused_rhs import device_scalars
    from bssn3d_b200.ozaki import OzakiDerivatives
    from oracle import ozaki_oracle as Z
    grid, U, dt = _state(n=12)
    Sd = device_scalars(_S(grid, dt), torch.device("cuda"))
    oz = OzakiDerivatives(U.shape[1:], k)
    got = oz.derivatives(torch.from_numpy(U).cuda(), Sd, ko_sigma=0.1, ko_order=ko_order).cpu().numpy()
    oz.check()
    want = Z.bundle(U, (grid.dx, grid.dy, grid.dz), k, ko_sigma=0.1, ko_order=ko_order)
    bad = [s for s in range(162) if not np.array_equal(got[s], want[s])]
    assert not bad, bad[:10]
