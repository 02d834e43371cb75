"""The q = 1/10 Brill-Lindquist workload (puncture masses 0.909 at x = -0.5
and 0.0909 at x = +5 on [-8,8]^3): 10 RK4 steps on the GPU against the CPU
oracle, per field and on the interior Hamiltonian-constraint norm
(3D/src/bssn3d/constraints.py:53-62), at a size the oracle finishes in
seconds; and at the full 128^3 size through properties that do not depend on
size: unit conformal determinant and traceless A~ after enforcement, finite
state, and the fused GPU constraint norms against the oracle's on the same
final state."""

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu


def _S(grid, dt, t=0.0):
    from bssn3d_b200.fused_rhs import pack_S
    return pack_S(2.0, 0.06, dt, grid.dx, 0.6, 20.0, t, (1, 1, 1, 1), (1, 0), grid.dy, grid.dz)


def test_ten_steps_vs_oracle_and_hamiltonian_norm():
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.constraints import ConstraintSolver
    from bssn3d_b200.evolve import BSSNEvolution
    from bssn3d_b200.state import BSSNState
    grid, U, dt = ID.workload(1, n=24)
    evo = BSSNEvolution(grid, ko_sigma=0.1, bc="none", ko_order=6)
    out = evo.evolve(BSSNState(torch.from_numpy(U).cuda()), dt, 10).data
    ref = U
    S = _S(grid, dt)
    for s in range(10):
        ref = O.rk4_step(ref, S, ko_sigma=0.1, ko_order=6)
        S[6] = S[6] + dt
    got = out.cpu().numpy()
    assert np.isfinite(got).all()
    assert O.normwise_rel_grouped(got, ref).max() < 1e-11
    h_gpu, m_gpu = ConstraintSolver(grid).l2(out)
    h_ref, m_ref = O.constraint_norms(ref, grid.dx, grid.dy, grid.dz, grid.ng)
    assert h_gpu == pytest.approx(h_ref, rel=1e-10)
    assert m_gpu == pytest.approx(m_ref, rel=1e-9)


@pytest.mark.slow
def test_full_size_ten_steps_properties():
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.constraints import ConstraintSolver
    from bssn3d_b200.evolve import BSSNEvolution
    from bssn3d_b200.state import BSSNState
    grid, U, dt = ID.workload(1)
    assert grid.shape == (134, 134, 134)
    evo = BSSNEvolution(grid, ko_sigma=0.1, bc="none", ko_order=6)
    out = evo.evolve(BSSNState(torch.from_numpy(U).cuda()), dt, 10).data
    g = out[3:9]
    det = g[0] * (g[3] * g[5] - g[4] ** 2) - g[1] * (g[1] * g[5] - g[4] * g[2]) + g[2] * (g[1] * g[4] - g[3] * g[2])
    assert float((det - 1.0).abs().max()) < 1e-12
    a = out[12:18]
    iu = torch.stack([g[3] * g[5] - g[4] ** 2, g[2] * g[4] - g[1] * g[5], g[1] * g[4] - g[2] * g[3],
                      g[0] * g[5] - g[2] ** 2, g[1] * g[2] - g[0] * g[4], g[0] * g[3] - g[1] ** 2])
    tr = iu[0] * a[0] + iu[3] * a[3] + iu[5] * a[5] + 2 * (iu[1] * a[1] + iu[2] * a[2] + iu[4] * a[4])
    assert float(tr.abs().max()) < 1e-10 * max(float(a.abs().max()), 1e-300)
    assert bool(torch.isfinite(out).all())
    h_gpu, m_gpu = ConstraintSolver(grid).l2(out)
    h_ref, m_ref = O.constraint_norms(out.cpu().numpy(), grid.dx, grid.dy, grid.dz, grid.ng)
    assert h_gpu == pytest.approx(h_ref, rel=1e-10)
    assert m_gpu == pytest.approx(m_ref, rel=1e-9)
