"""The reference's evolution and constraint checks on the GPU path:
3D/tests/integration/test_bssn_apples.py:40-82 (conformal algebra preserved,
noise stays bounded, gauge wave stays bounded) and
3D/tests/unit/test_bssn_constraints.py:23-56 (discrete constraints of the
exact gauge-wave data converge at order > 5.5; flat space gives zero)."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


def _det_trace(d):
    g = [d[3 + i] for i in range(6)]
    det = (g[0] * (g[3] * g[5] - g[4] ** 2) - g[1] * (g[1] * g[5] - g[4] * g[2])
           + g[2] * (g[1] * g[4] - g[3] * g[2]))
    iuxx, iuyy, iuzz = g[3] * g[5] - g[4] ** 2, g[0] * g[5] - g[2] ** 2, g[0] * g[3] - g[1] ** 2
    iuxy, iuxz, iuyz = g[2] * g[4] - g[1] * g[5], g[1] * g[4] - g[2] * g[3], g[1] * g[2] - g[0] * g[4]
    a = [d[12 + i] for i in range(6)]
    trA = (iuxx * a[0] + iuyy * a[3] + iuzz * a[5]
           + 2 * (iuxy * a[1] + iuxz * a[2] + iuyz * a[4])) / det
    return det, trA


def _evolve(N, data, nsteps):
    from bssn3d_b200.evolve import BSSNEvolution
    from bssn3d_b200.grid import Grid
    from bssn3d_b200.state import BSSNState
    g = Grid.from_domain(N, order=6)
    ev = BSSNEvolution(g, order=6, ko_sigma=0.1, bc="periodic")
    U = torch.from_numpy(data(g)).cuda()
    return g, U, ev.evolve(BSSNState(U), dt=0.25 * g.dx, nsteps=nsteps).data


def test_conformal_algebra_preserved():
    from bssn3d_b200 import initial_data as ID
    _, _, s = _evolve(12, lambda g: ID.gauge_wave(g, amplitude=0.01), 8)
    det, trA = _det_trace(s)
    assert bool(torch.isfinite(s).all())
    assert float((det - 1.0).abs().max()) < 1e-12
    assert float(trA.abs().max()) < 1e-10
    assert float(s[1].min()) > 0.0


def test_robust_stability_bounded():
    from bssn3d_b200 import initial_data as ID
    amp = 1e-8
    g, _, s = _evolve(12, lambda g: ID.robust_stability(g, amp=amp, seed=1), 40)
    dev = float((s - torch.from_numpy(ID.minkowski(g)).cuda()).abs().max())
    assert bool(torch.isfinite(s).all())
    assert dev < 1e-4


def test_gauge_wave_dynamically_stable():
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.constraints import ConstraintSolver
    g, _, s = _evolve(16, lambda g: ID.gauge_wave(g, amplitude=0.01), 40)
    H, M = ConstraintSolver(g, order=6).l2(s)
    assert bool(torch.isfinite(s).all())
    assert float(s[0].abs().max()) < 2.0
    assert H < 0.5 and M < 0.5


@pytest.fixture(scope="module")
def orders():
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.constraints import ConstraintSolver
    from bssn3d_b200.grid import Grid
    Ns = [24, 32, 48]
    H, M = [], []
    for N in Ns:
        g = Grid.from_domain(N, order=6, lo=-0.5, hi=0.5)
        h, m = ConstraintSolver(g, order=6).l2(ID.gauge_wave(g, amplitude=0.01))
        H.append(h)
        M.append(m)
    r = np.log(Ns[-1] / Ns[-2])
    return np.log(H[-2] / H[-1]) / r, np.log(M[-2] / M[-1]) / r


def test_hamiltonian_converges_at_fd_order(orders):
    assert orders[0] > 5.5


def test_momentum_converges_at_fd_order(orders):
    assert orders[1] > 5.5


def test_minkowski_constraints_vanish():
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.constraints import ConstraintSolver
    from bssn3d_b200.grid import Grid
    g = Grid.from_domain(16, order=6)
    H, M = ConstraintSolver(g, order=6).l2(ID.minkowski(g))
    assert H < 1e-13 and M < 1e-13
