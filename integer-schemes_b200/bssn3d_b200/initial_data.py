"""Initial data for the BSSN path (host-side input synthesis, numpy float64).

* ``minkowski``, ``robust_stability`` and ``gauge_wave`` restate
  3D/src/bssn3d/initial_data.py:28, :58-69 and :72-135 (the harmonic gauge
  wave is the one the reference's fused-kernel test uses,
  test_bssn_fused_cuda.py:41-49).
* ``brill_lindquist`` is new: the reference has no puncture data
  (initial_data.py:1-14). It builds the two-puncture conformally flat data the
  benchmark workloads are quoted on: psi = 1 + m1/(2 r1) + m2/(2 r2) with r
  floored at dx/2, chi = psi^-4, alpha = psi^-2, beta = B = Gt = K = At = 0,
  and gt_ij = delta_ij plus seeded N(0, sigma) noise on the off-diagonals,
  rescaled to unit determinant.

Every generator returns a ``(24, Sx, Sy, Sz)`` numpy array; move it to the
GPU with ``torch.from_numpy(a).cuda()``.
"""

from __future__ import annotations

from dataclasses import dataclass
from typing import Tuple

import numpy as np

from .grid import Grid
from .state import (ALPHA, AT0, AT3, AT5, CHI, GT0, GT1, GT2, GT3, GT4, GT5,
                    GTILDE0, K, NUM_VARS)


def minkowski(grid: Grid) -> np.ndarray:
    data = np.zeros((NUM_VARS,) + grid.shape)
    for k in (ALPHA, CHI, GT0, GT3, GT5):
        data[k] = 1.0
    return data


def robust_stability(grid: Grid, amp: float = 1.0e-10, seed: int = 0) -> np.ndarray:
    """Minkowski plus uniform noise in [-amp, amp) on all 24 fields
    (initial_data.py:58-69). The noise is drawn with
    ``numpy.random.default_rng(seed)``, not JAX's PRNG, so the samples differ
    from the reference's for the same seed; the test it serves (noise must
    not grow) depends only on the amplitude."""
    rng = np.random.default_rng(seed)
    return minkowski(grid) + rng.uniform(-amp, amp, size=(NUM_VARS,) + grid.shape)


def gauge_wave(grid: Grid, amplitude: float = 0.01, wavelength: float = None,
               axis: int = 0) -> np.ndarray:
    """1D harmonic gauge wave along ``axis`` at t = 0 (initial_data.py:72-135)."""
    coords = (grid.x, grid.y, grid.z)[axis]
    if wavelength is None:
        wavelength = float(coords[-grid.ng - 1] - coords[grid.ng]) + (grid.dx, grid.dy, grid.dz)[axis]
    X, Y, Z = grid.mesh()
    coord = (X, Y, Z)[axis]
    k = 2.0 * np.pi / wavelength
    phase = k * coord
    A = amplitude
    H = 1.0 - A * np.sin(phase)
    dH_dx = -A * k * np.cos(phase)
    dH_dt = -dH_dx
    sqrtH = np.sqrt(H)
    Kxx = -dH_dt / (2.0 * sqrtH)
    Ktrace = Kxx / H
    chi = H ** (-1.0 / 3.0)
    gt_wave = H ** (2.0 / 3.0)
    gt_trans = chi
    At_wave = chi * (Kxx - (1.0 / 3.0) * H * Ktrace)
    At_trans = chi * (0.0 - (1.0 / 3.0) * 1.0 * Ktrace)
    Gt_wave = (2.0 / 3.0) * H ** (-5.0 / 3.0) * dH_dx
    data = np.zeros((NUM_VARS,) + grid.shape)
    data[ALPHA] = sqrtH
    data[CHI] = chi
    data[K] = Ktrace
    gt_diag = (GT0, GT3, GT5)
    at_diag = (AT0, AT3, AT5)
    for a in range(3):
        data[gt_diag[a]] = gt_wave if a == axis else gt_trans
        data[at_diag[a]] = At_wave if a == axis else At_trans
    data[GTILDE0 + axis] = Gt_wave
    return data


@dataclass(frozen=True)
class Puncture:
    mass: float
    position: Tuple[float, float, float]


def brill_lindquist(grid: Grid, punctures, noise_sigma: float = 1e-8,
                    seed: int = 0) -> np.ndarray:
    """Brill-Lindquist punctures on ``grid`` (conformally flat, time-symmetric).

    ``r`` is floored at ``dx/2`` so a puncture sitting on a node stays finite.
    The off-diagonal metric noise is drawn from ``numpy.random.default_rng(seed)``
    in the order gt1, gt2, gt4 over the whole padded array; the metric is then
    rescaled by det^(-1/3) so det(gt) = 1.
    """
    X, Y, Z = grid.mesh()
    psi = np.ones(grid.shape)
    rmin = 0.5 * grid.dx
    for p in punctures:
        px, py, pz = p.position
        r = np.sqrt((X - px) ** 2 + (Y - py) ** 2 + (Z - pz) ** 2)
        r = np.maximum(r, rmin)
        psi = psi + p.mass / (2.0 * r)
    data = np.zeros((NUM_VARS,) + grid.shape)
    data[CHI] = psi ** -4
    data[ALPHA] = psi ** -2
    rng = np.random.default_rng(seed)
    g = np.zeros((6,) + grid.shape)
    g[0] = 1.0
    g[3] = 1.0
    g[5] = 1.0
    for k in (1, 2, 4):
        g[k] = noise_sigma * rng.standard_normal(grid.shape)
    det = g[0] * (g[3] * g[5] - g[4] * g[4]) - g[1] * (g[1] * g[5] - g[4] * g[2]) + \
        g[2] * (g[1] * g[4] - g[3] * g[2])
    scale = det ** (-1.0 / 3.0)
    for k, f in enumerate((GT0, GT1, GT2, GT3, GT4, GT5)):
        data[f] = g[k] * scale
    return data


# The benchmark workloads (seed = 20261203 + workload index).
def workload(index: int, n: int = None, ng: int = 3):
    """(grid, state, dt) of the numbered Brill-Lindquist workload.

    0: 64^3 interior on [-4,4]^3, m1 = m2 = 0.5 at x = -1.5, +1.5
    1: 128^3 on [-8,8]^3, m1 = 0.909 at x = -0.5, m2 = 0.0909 at x = +5.0 (q = 1/10)
    2: 192^3 on [-8,8]^3 with the index-1 punctures
    ``n`` overrides the interior size (same domain); dt = 0.25 dx.
    """
    if index == 0:
        N, lo, hi = 64, -4.0, 4.0
        punct = [Puncture(0.5, (-1.5, 0.0, 0.0)), Puncture(0.5, (1.5, 0.0, 0.0))]
    elif index in (1, 2):
        N, lo, hi = (128 if index == 1 else 192), -8.0, 8.0
        punct = [Puncture(0.909, (-0.5, 0.0, 0.0)), Puncture(0.0909, (5.0, 0.0, 0.0))]
    else:
        raise ValueError(f"unknown workload {index}")
    if n is not None:
        N = n
    grid = Grid.from_domain(N, lo=lo, hi=hi, ng=ng)
    state = brill_lindquist(grid, punct, noise_sigma=1e-8, seed=20261203 + index)
    return grid, state, 0.25 * grid.dx
