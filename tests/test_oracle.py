"""The CPU oracle pinned against the reference: golden fixtures made from the
reference's own compiled algebra, the reference's own known-answer tests
(Minkowski, bit-compare seeds) and stencil properties.

Mirrors 3D/tests/integration/test_bssn_oracle.py:22-33 (bit-compare, rel
< 1e-12), 3D/tests/unit/test_bssn_rhs.py:62-65 (Minkowski < 1e-12) and
3D/tests/unit/test_derivatives.py (stencil exactness).
"""

import numpy as np
import pytest

from conftest import GOLDEN
from oracle import oracle as O


def _pointwise_rel(a, b):
    return np.abs(a - b) / np.maximum(np.maximum(np.abs(a), np.abs(b)), 1e-12)


def test_algebra_golden_points():
    g = np.load(GOLDEN / "algebra_points.npz")
    out = O.rhs_algebra(g["F"], g["D"], g["S"])
    assert _pointwise_rel(out, g["OUT"]).max() < 1e-12


def test_algebra_vs_compiled_reference_many_points():
    if not O.have_ref():
        pytest.skip("oracle/_ref not built (reference tree absent)")
    rng = np.random.default_rng(7)
    n = 4096
    F = np.zeros((24, n))
    F[:] = 0.1 * rng.uniform(-1, 1, F.shape)
    F[0] += 1.0
    F[1] = 0.05 + rng.uniform(0, 1, n)          # chi down to 0.05 (near-puncture values)
    for k in (3, 6, 8):
        F[k] += 1.0
    D = 0.5 * rng.standard_normal((138, n))
    S = np.array([2.0, 0.06, 0.03, 0.125, 0.6, 20, 0.4, 1, 1, 1, 1, 1, 0, 0.125, 0.125, 0.125])
    a = O.rhs_algebra(F, D, S)
    b = O.ref_rhs_algebra(F, D, S)
    assert O.normwise_rel(a, b).max() < 1e-13


def test_minkowski_rhs_vanishes():
    shape = (10, 11, 12)
    F = np.zeros((24,) + shape)
    for k in (0, 1, 3, 6, 8):
        F[k] = 1.0
    S = np.array([2.0, 0.06, 0.03, 0.1, 0.6, 20, 0.0, 1, 1, 1, 1, 1, 0, 0.1, 0.1, 0.1])
    S[4] = 0.0  # SSL off; with alpha = chi = 1 it vanishes anyway
    out = O.rhs(F, S)
    assert np.abs(out).max() < 1e-12


def test_bl_small_rhs_and_step():
    g = np.load(GOLDEN / "bl_small.npz")
    out = O.rhs(g["U"], g["S"])
    assert O.normwise_rel(out, g["rhs"]).max() < 1e-13
    step = O.rk4_step(g["U"], g["S"], ko_sigma=float(g["ko_sigma"]), ko_order=int(g["ko_order"]))
    # the evolved state is measured per tensor (its off-diagonal metric entries
    # are 1e-8 noise); the taps here are fused multiply-adds, the fixture's
    # separately rounded, so the two differ by rounding only
    assert O.normwise_rel_grouped(step, g["step"]).max() < 5e-14


def test_gauge_wave_rhs():
    g = np.load(GOLDEN / "gauge_wave_rhs.npz")
    out = O.rhs(g["U"], g["S"])
    # fields whose RHS is identically zero for this data compare in absolute terms
    err = np.abs(out - g["rhs"]).reshape(24, -1).max(axis=1)
    scale = np.abs(g["rhs"]).reshape(24, -1).max(axis=1)
    assert np.all(err <= 1e-13 * np.maximum(scale, 1.0))


def test_first_derivative_exact_on_polynomials():
    # 6th-order centred stencils differentiate polynomials of degree <= 6 exactly
    Sx, Sy, Sz = 12, 13, 14
    h = (0.1, 0.07, 0.13)
    x = np.arange(Sx)[:, None, None] * h[0]
    y = np.arange(Sy)[None, :, None] * h[1]
    z = np.arange(Sz)[None, None, :] * h[2]
    f = 0.3 * x ** 5 - x ** 2 * y ** 3 + 2 * y * z ** 4 + z ** 6 + x * y * z
    F = np.zeros((24, Sx, Sy, Sz))
    F[0] = f
    D = O.derivatives(F, *h)
    sl = (slice(3, -3),) * 3
    fx = 1.5 * x ** 4 - 2 * x * y ** 3 + y * z
    fz = 8 * y * z ** 3 + 6 * z ** 5 + x * y
    fxy = -6 * x * y ** 2 + z
    fzz = 24 * y * z ** 2 + 30 * z ** 4
    np.testing.assert_allclose(D[0][sl], np.broadcast_to(fx, f.shape)[sl], rtol=0, atol=1e-9)
    np.testing.assert_allclose(D[2][sl], np.broadcast_to(fz, f.shape)[sl], rtol=0, atol=1e-9)
    np.testing.assert_allclose(D[72 + 1][sl], np.broadcast_to(fxy, f.shape)[sl], rtol=0, atol=1e-8)
    np.testing.assert_allclose(D[72 + 5][sl], np.broadcast_to(fzz, f.shape)[sl], rtol=0, atol=1e-8)


def test_edge_clamp_matches_composed_padding():
    # mixed derivative at the corner: clamping both axes == composing the per-axis pads
    rng = np.random.default_rng(3)
    F = np.zeros((24, 7, 8, 9))
    F[1] = rng.standard_normal((7, 8, 9))
    D = O.derivatives(F, 0.1, 0.2, 0.3)
    c1 = np.array([-1, 9, -45, 0, 45, -9, 1]) / 60.0

    def d1(u, h, axis):
        pad = [(3, 3) if a == axis else (0, 0) for a in range(3)]
        p = np.pad(u, pad, mode="edge")
        n = u.shape[axis]
        return sum((c1[k] / h) * np.take(p, range(k, k + n), axis=axis) for k in range(7))

    ref = d1(d1(F[1], 0.1, 0), 0.2, 1)
    np.testing.assert_allclose(D[72 + 6 * 1 + 1], ref, rtol=0, atol=1e-11)


def test_ko_annihilates_low_polynomials():
    Sx = Sy = Sz = 14
    x = np.arange(Sx)[:, None, None] * 0.1
    F = np.zeros((24, Sx, Sy, Sz))
    F[5] = np.broadcast_to(1 + x + x ** 2 + x ** 5, (Sx, Sy, Sz))
    K6 = O.ko(F, 0.1, 0.1, 0.1, 0.3, 6)
    K8 = O.ko(F, 0.1, 0.1, 0.1, 0.3, 8)
    sl = (slice(4, -4),) * 3
    assert np.abs(K6[5][sl]).max() < 1e-10
    assert np.abs(K8[5][sl]).max() < 1e-10


def test_enforce_unit_det_and_traceless():
    rng = np.random.default_rng(5)
    F = np.zeros((24, 5, 5, 5))
    F[:] = 0.05 * rng.standard_normal(F.shape)
    for k in (3, 6, 8):
        F[k] += 1.0
    F[1] = -1.0  # below the floor
    E = O.enforce(F)
    g = E[3:9]
    det = g[0] * (g[3] * g[5] - g[4] ** 2) - g[1] * (g[1] * g[5] - g[4] * g[2]) + g[2] * (g[1] * g[4] - g[3] * g[2])
    np.testing.assert_allclose(det, 1.0, atol=1e-14)
    assert np.all(E[1] == 1e-4)


def test_periodic_sync():
    rng = np.random.default_rng(9)
    F = rng.standard_normal((24, 12, 12, 12))
    P = O.periodic_sync(F, 3)
    np.testing.assert_array_equal(P[:, :3], P[:, 6:9])
    np.testing.assert_array_equal(P[:, -3:], P[:, 3:6])
    np.testing.assert_array_equal(P[:, :, :, :3], P[:, :, :, 6:9])


def test_constraints_golden():
    g = np.load(GOLDEN / "bl_small.npz")
    S = g["S"]
    H, M = O.constraints(g["U"], S[13], S[14], S[15])
    assert np.abs(H - g["H"]).max() <= 1e-13 * np.abs(g["H"]).max()
    assert np.abs(M - g["M"]).max() <= 1e-13 * max(np.abs(g["M"]).max(), 1e-300) or np.abs(g["M"]).max() == 0


def test_constraints_vs_compiled_physcon():
    if not O.have_physcon():
        pytest.skip("oracle/_ref not built (reference tree absent)")
    rng = np.random.default_rng(21)
    n = 2048
    F = 0.1 * rng.uniform(-1, 1, (24, n))
    F[0] += 1.0
    F[1] = 0.05 + rng.uniform(0, 1, n)
    for k in (3, 6, 8):
        F[k] += 1.0
    D = 0.5 * rng.standard_normal((138, n))
    H, M = O.constraints_algebra(F, D)
    Hr, Mr = O.ref_constraints_algebra(F, D)
    assert np.abs(H - Hr).max() <= 1e-13 * np.abs(Hr).max()
    assert np.abs(M - Mr).max() <= 1e-13 * np.abs(Mr).max()


def test_oracle_algebra_on_the_reference_vector_recipe():
    """The oracle against the reference's compiled algebra on the inputs of its
    algebra-only vector file (gen_algebra_cuda.py:99-140), 2^16 of its 2^18 points."""
    if not O.have_ref():
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(1)
    n = 1 << 16
    F = np.empty((24, n))
    for f in range(24):
        F[f] = (1.0 if f in (0, 1, 3, 6, 8) else 0.0) + 0.03 * rng.standard_normal(n)
    D = 0.03 * rng.standard_normal((138, n))
    S = np.array([2.0, 0.06, 0.01, 0.1, 0.6, 20.0, 0.0, 1, 1, 1, 1, 1, 0, 0.1, 0.1, 0.1])
    assert O.normwise_rel(O.rhs_algebra(F, D, S), O.ref_rhs_algebra(F, D, S)).max() < 1e-13
