"""The CPU restatement of the Ozaki INT8 bundle (oracle/ozaki_oracle.py), no
GPU: at k = 8 it reproduces the float64 oracle's 138 derivatives and KO sums
to rounding on the field's scale, the error grows as k falls, and a field of
few significant bits is split exactly (its stencil sums equal the float64
ones whenever those are exact too)."""

import numpy as np
import pytest

from oracle import oracle as O
from oracle import ozaki_oracle as Z


def _state(n=10):
    from bssn3d_b200 import initial_data as ID
    grid, U, dt = ID.workload(1, n=n)
    return grid, U


def _scales(U, h):
    fmax = np.abs(U.reshape(24, -1)).max(axis=1)
    sc = np.empty(162)
    for f in range(24):
        sc[3 * f:3 * f + 3] = fmax[f] / h
        sc[138 + f] = fmax[f] / h
    for m, f in enumerate(Z.D2_FIELDS):
        sc[72 + 6 * m:72 + 6 * m + 6] = fmax[f] / h ** 2
    return np.maximum(sc, 1e-300)


@pytest.mark.parametrize("ko_order", [6, 8])
def test_bundle_converges_to_float64(ko_order):
    grid, U = _state()
    h = grid.dx
    ref = np.concatenate([O.derivatives(U, h, h, h), O.ko(U, h, h, h, 0.1, ko_order)])
    sc = _scales(U, h)
    errs = []
    for k in (4, 6, 8):
        D = Z.bundle(U, h, k, ko_sigma=0.1, ko_order=ko_order)
        assert np.isfinite(D).all()
        errs.append(float((np.abs(D - ref).reshape(162, -1).max(axis=1) / sc).max()))
    assert errs[2] < 1e-13
    assert errs[0] > errs[1] > errs[2]


def test_exact_split_of_short_values():
    # values on a 2^-10 lattice need few digits: at k = 4 (28 bits) the split is exact
    rng = np.random.default_rng(1)
    F = rng.integers(-512, 512, size=(1, 12, 13, 14)).astype(np.float64) / 1024.0
    d1, d2, _ = Z.ozaki_pass(F[0], 2, 4, 1.0, True)
    # exact integer sums, one rounding in the final scaling, like the float64 stencil on exact data
    C1 = np.array([-1, 9, -45, 0, 45, -9, 1]) / 60.0
    P = np.pad(F[0], ((0, 0), (0, 0), (3, 3)), mode="edge")
    want = sum(C1[j] * P[:, :, j:j + 14] for j in range(7))
    np.testing.assert_allclose(d1, want, rtol=0, atol=1e-15)


def test_covered_box_with_core():
    grid, U = _state(n=10)
    h = grid.dx
    full = Z.bundle(U, h, 6, ko_sigma=0.1)
    cored = Z.bundle(U, h, 6, ko_sigma=0.1, core=3)
    I = (slice(None),) + (slice(3, -3),) * 3
    assert np.isfinite(cored[I]).all()
    # derivatives at the interior of a cored pass are those of the whole-array pass
    # up to the window exponents, which depend on where the 16-output groups start
    sc = _scales(U, h)[:, None]
    assert (np.abs(cored[I] - full[I]).reshape(162, -1) / sc).max() < 1e-9
