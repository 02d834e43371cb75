"""MSRK integrator on the GPU (bssn_b200_msrk_stage, BSSNEvolution with
integrator="rk4_2_1"/"rk4_2_2"): one step and whole runs against the oracle's
restatement of evolve.py:139-183, and the reference's own MSRK checks
(3D/tests/integration/test_msrk_evolve.py:33-72): agreement with RK4 to
truncation, 4th-order agreement, stability at CFL 0.1 / KO 0.4."""

import ctypes

import numpy as np
import pytest
import torch

from oracle import oracle as O

pytestmark = pytest.mark.gpu

CFL, KO = 0.1, 0.4


def _S(grid, dt, t=0.0):
    from bssn3d_b200.fused_rhs import pack_S
    return pack_S(2.0, 0.06, dt, grid.dx, 0.6, 20.0, t, (1, 1, 1, 1), (1, 0), grid.dy, grid.dz)


def _rms(a):
    return float(torch.sqrt(torch.mean(a ** 2)))


def _evo(grid, integ, ko=KO, bc="periodic", ko_order=8):
    from bssn3d_b200.evolve import BSSNEvolution
    return BSSNEvolution(grid, ko_sigma=ko, bc=bc, integrator=integ, ko_order=ko_order)


@pytest.mark.parametrize("method", ["rk4_2_1", "rk4_2_2"])
def test_msrk_step_vs_oracle(method):
    from bssn3d_b200 import initial_data as ID, msrk
    from bssn3d_b200.state import BSSNState
    grid, U, dt = ID.workload(1, n=20)
    S = _S(grid, dt, t=0.3)
    Sp = S.copy()
    Sp[6] -= dt
    fprev = O.rate(U, Sp, ko_sigma=0.1, ko_order=6)   # a k0 from the previous step time
    evo = _evo(grid, method, ko=0.1, bc="none", ko_order=6)
    y, k = evo.msrk_step(BSSNState(torch.from_numpy(U).cuda()), torch.from_numpy(fprev).cuda(), 0.3, dt)
    y_ref, k_ref = O.msrk2_step(U, fprev, S, msrk.METHODS[method].coef, ko_sigma=0.1, ko_order=6)
    assert O.normwise_rel_grouped(y.data.cpu().numpy(), y_ref).max() < 1e-12
    assert O.normwise_rel_grouped(k.data.cpu().numpy(), k_ref).max() < 1e-11


@pytest.mark.parametrize("method,bc,ko_order", [("rk4_2_2", "periodic", 8), ("rk4_2_1", "none", 6)])
def test_msrk_evolve_vs_oracle(method, bc, ko_order):
    from bssn3d_b200 import initial_data as ID, msrk
    from bssn3d_b200.grid import Grid
    from bssn3d_b200.state import BSSNState
    g = Grid.from_domain(12, ko_order=ko_order)
    U = ID.gauge_wave(g, amplitude=0.01)
    dt = CFL * g.dx
    out = _evo(g, method, bc=bc, ko_order=ko_order).evolve(BSSNState(torch.from_numpy(U).cuda()), dt, 6)
    ref = O.msrk_evolve(U, _S(g, dt), msrk.METHODS[method].coef, 6, ko_sigma=KO, ko_order=ko_order,
                        periodic=(bc == "periodic"), ng=g.ng)
    assert O.normwise_rel_grouped(out.data.cpu().numpy(), ref).max() < 1e-11


def test_msrk_graph_replay_matches_eager():
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.state import BSSNState
    grid, U, dt = ID.workload(1, n=16)
    evo = _evo(grid, "rk4_2_2", ko=0.1, bc="none", ko_order=6)
    s = BSSNState(torch.from_numpy(U).cuda())
    a = evo.evolve(s, dt, 5, use_graph=True).data
    b = evo.evolve(s, dt, 5, use_graph=False).data
    assert torch.equal(a, b)
    one = evo.evolve(s, dt, 1).data
    rk4 = _evo(grid, "rk4", ko=0.1, bc="none", ko_order=6).evolve(s, dt, 1).data
    assert torch.equal(one, rk4)          # the first step is the RK4 startup step


def test_rk42_reproduces_rk4_to_truncation():
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.grid import Grid
    from bssn3d_b200.state import BSSNState
    grid = Grid.from_domain(16)
    ic = BSSNState(torch.from_numpy(ID.gauge_wave(grid, amplitude=0.01)).cuda())
    dt = CFL * grid.dx
    s4 = _evo(grid, "rk4").evolve(ic, dt, 40).data
    s2 = _evo(grid, "rk4_2_2").evolve(ic, dt, 40).data
    assert bool(torch.isfinite(s2).all())
    assert _rms(s2 - s4) / _rms(s4) < 1e-5


def test_agreement_is_fourth_order():
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.grid import Grid
    from bssn3d_b200.state import BSSNState
    grid = Grid.from_domain(16)
    ic = BSSNState(torch.from_numpy(ID.gauge_wave(grid, amplitude=0.01)).cuda())

    def gap(cfl, nsteps):
        dt = cfl * grid.dx
        s4 = _evo(grid, "rk4").evolve(ic, dt, nsteps).data
        s2 = _evo(grid, "rk4_2_2").evolve(ic, dt, nsteps).data
        return _rms(s2 - s4)

    assert gap(0.10, 20) / gap(0.05, 40) > 8.0


def test_stable_at_production_cfl_ko():
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.grid import Grid
    from bssn3d_b200.state import BSSNState
    grid = Grid.from_domain(16)
    ic = torch.from_numpy(ID.gauge_wave(grid, amplitude=0.01)).cuda()
    s = _evo(grid, "rk4_2_2").evolve(BSSNState(ic), CFL * grid.dx, 200).data
    assert bool(torch.isfinite(s).all())
    assert _rms(s) < 10.0 * _rms(ic)


def test_msrk_stage_rejects_bad_operands_without_launching():
    from bssn3d_b200 import _lib, msrk
    lib = _lib.load()
    n = 12
    U = torch.zeros(24, n, n, n, dtype=torch.float64, device="cuda")
    A, B, C, D = (torch.zeros_like(U) for _ in range(4))
    S = torch.zeros(16, dtype=torch.float64, device="cuda")
    coef = (ctypes.c_double * 9)(*msrk.METHODS["rk4_2_2"].coef)
    cp = ctypes.cast(coef, ctypes.c_void_p)
    p = lambda t: None if t is None else t.data_ptr()
    stream = torch.cuda.current_stream().cuda_stream

    def call(stage, u, y, acc, out, out2, out3, c=cp):
        return lib.bssn_b200_msrk_stage(stream, stage, p(u), p(y), p(acc), p(out), p(out2), p(out3),
                                        S.data_ptr(), c, 0.1, 6, 1e-4, 1e-4, n, n, n)

    before = A.clone()
    assert call(3, U, U, A, B, C, D) == _lib.EINVAL
    assert call(0, U, U, A, U, C, D) == _lib.EINVAL       # OUT aliases the stencil input
    assert call(0, U, U, A, B, B, D) == _lib.EINVAL       # stage-0 outputs not distinct
    assert call(0, U, U, A, B, C, None) == _lib.EINVAL    # OUT3 missing
    assert call(1, B, A, C, A, None, None) == _lib.EINVAL  # OUT aliases Y
    assert call(1, B, A, B, C, None, None) == _lib.EINVAL  # ACC aliases U
    assert call(0, U, U, A, B, C, D, c=None) == _lib.EINVAL
    bad = (ctypes.c_double * 9)(*([float("nan")] + [0.0] * 8))
    assert call(0, U, U, A, B, C, D, c=ctypes.cast(bad, ctypes.c_void_p)) == _lib.EINVAL
    assert "msrk_stage" in lib.bssn_b200_last_error().decode()
    torch.cuda.synchronize()
    assert torch.equal(A, before)


def test_captured_graph_keeps_its_tensors_alive():
    """A graph replays on fixed addresses: the tensors it was captured on must
    outlive it even when the caller drops them and the memory is reused."""
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.state import BSSNState
    grid, U, dt = ID.workload(1, n=16)
    evo = _evo(grid, "rk4_2_2", ko=0.1, bc="none", ko_order=6)
    U0 = torch.from_numpy(U).cuda()
    ref = evo.evolve(BSSNState(U0), dt, 6).data.clone()
    S = evo._S(0.0, dt, U0.device)
    KP, U1 = torch.empty_like(U0), U0.clone()
    evo._startup_inplace(U1, KP, S)
    evo._advance_time(S)
    g, Ug, _, _ = evo.capture_msrk(U1, S, KP)
    del KP, S
    junk = []
    for _ in range(5):
        junk.append(torch.full_like(U0, float("nan")))
        junk.append(torch.full((16,), float("nan"), dtype=torch.float64, device="cuda"))
        g.replay()
    assert torch.equal(Ug, ref)
