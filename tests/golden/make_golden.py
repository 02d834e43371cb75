"""Generate the golden fixtures in tests/golden/ from the reference's own
compiled BSSN algebra (oracle/_ref/libdendro_ref.so, built by
``make -C oracle ref`` from 3D/src/bssn3d/vendor/bssneqs_SSL_HD_dxsq.cpp where
it lies in the reference tree).

    python tests/golden/make_golden.py

Fixtures (numpy .npz, float64, exact):

* ``algebra_points.npz`` — the reference's single-point bit-compare inputs,
  seeds 0-4, drawn with the recipe of 3D/src/bssn3d/oracle.py:46-86
  (``numpy.random.default_rng(seed)``; one uniform draw per field in state
  order, then one per derivative in the reference's sorted derivative-name
  order) and the reference's scalars; outputs from the reference algebra.
* ``bl_small.npz`` — a Brill-Lindquist state (two punctures, 6^3 interior + 3
  ghosts on [-4,4]^3), its RHS (restated stencils + reference algebra), one
  RK4 step composed as in 3D/src/bssn3d/evolve.py:125-137 (KO sigma 0.1,
  order 6, enforcement) and its Hamiltonian/momentum constraints from the
  reference's compiled physcon block (oracle/_ref/libdendro_physcon.so).
* ``gauge_wave_rhs.npz`` — the harmonic gauge wave (amplitude 0.01, 8^3
  interior + 3 ghosts on [-1/2,1/2]^3) and its RHS, the data the reference's
  fused-kernel test uses (3D/tests/integration/test_bssn_fused_cuda.py:41-49).
"""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "integer-schemes_b200"))

from oracle import oracle as O  # noqa: E402
from bssn3d_b200 import initial_data as ID  # noqa: E402
from bssn3d_b200.grid import Grid  # noqa: E402
from bssn3d_b200.state import VAR_NAMES  # noqa: E402
from bssn3d_b200.fused_rhs import pack_S  # noqa: E402

OUT = Path(__file__).resolve().parent

G2_FIELDS = ["alpha", "chi", "gt0", "gt1", "gt2", "gt3", "gt4", "gt5", "beta0", "beta1", "beta2"]
PAIRS = [(0, 0), (0, 1), (0, 2), (1, 1), (1, 2), (2, 2)]


def deriv_names():
    """Derivative names in the reference's sorted order and their slot here."""
    g1 = sorted((a, f) for a in range(3) for f in VAR_NAMES)
    g2 = sorted((i, j, f) for (i, j) in PAIRS for f in G2_FIELDS)
    names, slots = [], []
    for a, f in g1:
        names.append(f"grad_{a}_{f}")
        slots.append(3 * VAR_NAMES.index(f) + a)
    for i, j, f in g2:
        names.append(f"grad2_{i}_{j}_{f}")
        slots.append(72 + 6 * G2_FIELDS.index(f) + PAIRS.index((i, j)))
    return names, slots


def reference_point(seed: int):
    rng = np.random.default_rng(seed)
    F = np.zeros(24)
    for k, name in enumerate(VAR_NAMES):
        if name in ("gt0", "gt3", "gt5"):
            F[k] = 1.0 + 0.1 * rng.uniform(-1, 1)
        elif name in ("gt1", "gt2", "gt4"):
            F[k] = 0.05 * rng.uniform(-1, 1)
        elif name == "chi":
            F[k] = 1.0 + 0.2 * rng.uniform(0, 1)
        elif name == "alpha":
            F[k] = 1.0 + 0.1 * rng.uniform(-1, 1)
        else:
            F[k] = 0.1 * rng.uniform(-1, 1)
    names, slots = deriv_names()
    D = np.zeros(138)
    for s in slots:
        D[s] = 0.05 * rng.uniform(-1, 1)
    S = pack_S(2.13, 0.06, 0.013, 0.027, 0.6, 20.0, 1.7, (1.10, 0.90, 1.20, 0.80),
               (1.00, 0.50), 0.027, 0.027)
    return F, D, S


def rk4_step_reference(U, S, ko_sigma, ko_order):
    """evolve.py:125-137 composed from the reference's compiled algebra."""
    dt, t = S[2], S[6]
    g = (S[13], S[14], S[15])

    def rate(Y, tt):
        S2 = S.copy()
        S2[6] = tt
        r = O.ref_rhs(Y, S2)
        return r + O.ko(Y, *g, ko_sigma, ko_order)

    k1 = rate(U, t)
    k2 = rate(U + 0.5 * dt * k1, t + 0.5 * dt)
    k3 = rate(U + 0.5 * dt * k2, t + 0.5 * dt)
    k4 = rate(U + dt * k3, t + dt)
    new = U + (dt / 6.0) * (k1 + 2 * k2 + 2 * k3 + k4)
    return O.enforce(new)


def main():
    if not O.have_ref():
        raise SystemExit("oracle/_ref/libdendro_ref.so missing: run `make -C oracle ref`")
    pts = [reference_point(s) for s in range(5)]
    F = np.stack([p[0] for p in pts], axis=1)
    D = np.stack([p[1] for p in pts], axis=1)
    S = pts[0][2]
    OUTP = O.ref_rhs_algebra(F, D, S)
    np.savez(OUT / "algebra_points.npz", F=F, D=D, S=S, OUT=OUTP, seeds=np.arange(5))

    grid, U, dt = ID.workload(0, n=6)
    S = pack_S(2.0, 0.06, dt, grid.dx, 0.6, 20.0, 0.0, (1, 1, 1, 1), (1, 0), grid.dy, grid.dz)
    rhs = O.ref_rhs(U, S)
    step = rk4_step_reference(U, S, 0.1, 6)
    Dv = O.derivatives(U, grid.dx, grid.dy, grid.dz)
    H, M = O.ref_constraints_algebra(U, Dv)
    np.savez(OUT / "bl_small.npz", U=U, S=S, rhs=rhs, step=step, ko_sigma=0.1, ko_order=6,
             H=H, M=M)

    g = Grid.from_domain(8, ng=3)
    W = ID.gauge_wave(g, amplitude=0.01)
    dtg = 0.25 * g.dx
    S = pack_S(2.0, 0.06, dtg, g.dx, 0.6, 20.0, 0.0, (1, 1, 1, 1), (1, 0), g.dy, g.dz)
    np.savez(OUT / "gauge_wave_rhs.npz", U=W, S=S, rhs=O.ref_rhs(W, S))
    print("wrote", sorted(p.name for p in OUT.glob("*.npz")))


if __name__ == "__main__":
    main()
