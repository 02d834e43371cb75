"""GPU parity: the sm_100a kernels, called through the C ABI, against the CPU
oracle and the golden fixtures made from the reference's compiled algebra.

Bars (FP64 path): per-field normwise relative error <= 1e-12, the bar of the
B200 build; the reference's own single-point bit-compare bar is pointwise
relative < 1e-12 (3D/tests/integration/test_bssn_oracle.py:22-33), its
device-derivative bar 1e-11 absolute on a default_rng(11) normal state
(3D/tests/integration/test_deriv_kernel.py:55-74).
"""

import numpy as np
import pytest
import torch

from conftest import GOLDEN
from oracle import oracle as O

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


def _lib():
    from bssn3d_b200 import _lib as L
    return L


def _S(dx, dy, dz, dt=0.03, t=0.0, **kw):
    from bssn3d_b200.fused_rhs import pack_S
    p = dict(eta=2.0, cahd_c=0.06, ssl_h=0.6, ssl_sigma=20.0, lmbda=(1, 1, 1, 1), lambda_f=(1, 0))
    p.update(kw)
    return pack_S(p["eta"], p["cahd_c"], dt, dx, p["ssl_h"], p["ssl_sigma"], t, p["lmbda"],
                  p["lambda_f"], dy, dz)


def _dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).to(DEV)


def _gpu_rhs(U, S):
    from bssn3d_b200.fused_rhs import rhs_tensor, device_scalars
    out = rhs_tensor(_dev(U), device_scalars(S, DEV))
    return out.cpu().numpy()


def _random_state(shape, seed, amp=0.05):
    rng = np.random.default_rng(seed)
    F = amp * rng.standard_normal((24,) + shape)
    for k in (0, 1, 3, 6, 8):
        F[k] += 1.0
    return F


# ---------------------------------------------------------------- algebra
def test_algebra_golden_points():
    g = np.load(GOLDEN / "algebra_points.npz")
    F, D, S = _dev(g["F"]), _dev(g["D"]), _dev(g["S"])
    out = torch.empty_like(F)
    L = _lib()
    rc = L.load().bssn_b200_rhs_algebra(None, F.data_ptr(), D.data_ptr(), S.data_ptr(),
                                        out.data_ptr(), F.shape[1])
    L.check(rc)
    torch.cuda.synchronize()
    o = out.cpu().numpy()
    rel = np.abs(o - g["OUT"]) / np.maximum(np.maximum(np.abs(o), np.abs(g["OUT"])), 1e-12)
    assert rel.max() < 1e-12


def test_algebra_random_points_vs_oracle():
    rng = np.random.default_rng(12)
    n = 10000
    F = 0.1 * rng.uniform(-1, 1, (24, n))
    F[0] += 1.0
    F[1] = 0.05 + rng.uniform(0, 1, n)
    for k in (3, 6, 8):
        F[k] += 1.0
    D = 0.5 * rng.standard_normal((138, n))
    S = _S(0.125, 0.125, 0.125, t=0.4)
    Fd, Dd, Sd = _dev(F), _dev(D), _dev(S)
    out = torch.empty_like(Fd)
    L = _lib()
    L.check(L.load().bssn_b200_rhs_algebra(None, Fd.data_ptr(), Dd.data_ptr(), Sd.data_ptr(),
                                           out.data_ptr(), n))
    torch.cuda.synchronize()
    assert O.normwise_rel(out.cpu().numpy(), O.rhs_algebra(F, D, S)).max() < 1e-13


# ------------------------------------------------------------ derivatives
@pytest.mark.parametrize("ko_order,ng", [(6, 3), (8, 4)])
def test_derivatives_vs_oracle(ko_order, ng):
    from bssn3d_b200.fused_rhs import derivatives, device_scalars
    shape = (16 + 2 * ng, 16 + 2 * ng, 16 + 2 * ng)
    rng = np.random.default_rng(11)
    F = rng.standard_normal((24,) + shape)
    h = (0.0625, 0.0625, 0.0625)
    S = _S(*h)
    D = derivatives(_dev(F), device_scalars(S, DEV), ko_sigma=0.1, ko_order=ko_order).cpu().numpy()
    ref = O.derivatives(F, *h)
    # the reference's bar is 1e-11 absolute; the taps here are the reference's
    # own IEEE operations in the reference's order, so the bundle is bit-exact
    np.testing.assert_array_equal(D[:138], ref)
    ko = O.ko(F, *h, 0.1, ko_order)
    np.testing.assert_array_equal(D[138:], ko)


def test_derivatives_ragged_shape():
    from bssn3d_b200.fused_rhs import derivatives, device_scalars
    F = _random_state((7, 9, 19), 4, amp=1.0)
    h = (0.1, 0.2, 0.05)
    D = derivatives(_dev(F), device_scalars(_S(*h), DEV)).cpu().numpy()
    ref = O.derivatives(F, *h)
    np.testing.assert_array_equal(D, ref)


# -------------------------------------------------------------------- rhs
def test_rhs_bl_golden():
    g = np.load(GOLDEN / "bl_small.npz")
    out = _gpu_rhs(g["U"], g["S"])
    assert O.normwise_rel(out, g["rhs"]).max() < 1e-12


def test_rhs_gauge_wave_golden():
    g = np.load(GOLDEN / "gauge_wave_rhs.npz")
    out = _gpu_rhs(g["U"], g["S"])
    err = np.abs(out - g["rhs"]).reshape(24, -1).max(axis=1)
    scale = np.abs(g["rhs"]).reshape(24, -1).max(axis=1)
    assert np.all(err <= 1e-12 * np.maximum(scale, 1.0))
    # the reference's own fused-vs-verbatim bar (test_bssn_fused_cuda.py:41-49)
    assert err.max() <= 1e-8


@pytest.mark.parametrize("shape", [(20, 20, 20), (13, 27, 35), (4, 5, 40), (40, 44, 50)])
def test_rhs_random_state_vs_oracle(shape):
    F = _random_state(shape, sum(shape))
    S = _S(0.1, 0.11, 0.09, t=0.7)
    assert O.normwise_rel(_gpu_rhs(F, S), O.rhs(F, S)).max() < 1e-12


def test_rhs_minkowski_vanishes():
    F = np.zeros((24, 18, 18, 18))
    for k in (0, 1, 3, 6, 8):
        F[k] = 1.0
    out = _gpu_rhs(F, _S(0.1, 0.1, 0.1))
    assert np.abs(out).max() < 1e-12


def test_rhs_deterministic():
    F = _random_state((22, 22, 22), 1)
    S = _S(0.1, 0.1, 0.1)
    a = _gpu_rhs(F, S)
    b = _gpu_rhs(F, S)
    np.testing.assert_array_equal(a, b)


def test_cuda_fused_algebra_dict_interface():
    from bssn3d_b200.fused_rhs import cuda_fused_algebra
    from bssn3d_b200.state import FIELD_INPUTS, OUTPUT_FIELDS
    F = _random_state((12, 12, 12), 2)
    Fd = {name: _dev(F[k]) for k, name in enumerate(FIELD_INPUTS)}
    out = cuda_fused_algebra(Fd, 0.1, 0.1, 0.1, 2.0, (1, 1, 1, 1), (1, 0), 0.06, 0.025, 0.6, 20.0, 0.0)
    assert list(out) == OUTPUT_FIELDS
    ref = O.rhs(F, _S(0.1, 0.1, 0.1, dt=0.025))
    got = np.stack([out[n].cpu().numpy() for n in OUTPUT_FIELDS])
    assert O.normwise_rel(got, ref).max() < 1e-12


# --------------------------------------------------------------- RK4 step
def test_rk4_step_golden():
    from bssn3d_b200.evolve import BSSNEvolution
    from bssn3d_b200.grid import Grid
    from bssn3d_b200.state import BSSNState
    g = np.load(GOLDEN / "bl_small.npz")
    S = g["S"]
    grid = Grid.from_domain(6, lo=-4.0, hi=4.0, ng=3)
    evo = BSSNEvolution(grid, ko_sigma=float(g["ko_sigma"]), bc="none", ko_order=int(g["ko_order"]))
    new = evo.step(BSSNState(_dev(g["U"])), 0.0, float(S[2])).data.cpu().numpy()
    assert O.normwise_rel_grouped(new, g["step"]).max() < 1e-12


@pytest.mark.parametrize("ko_order,ng,bc", [(6, 3, "none"), (8, 4, "none"), (6, 3, "periodic")])
def test_evolve_vs_oracle(ko_order, ng, bc):
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.evolve import BSSNEvolution
    from bssn3d_b200.grid import Grid
    from bssn3d_b200.state import BSSNState
    grid = Grid.from_domain(12, lo=-4.0, hi=4.0, ng=ng)
    U = ID.brill_lindquist(grid, [ID.Puncture(0.5, (-1.0, 0.0, 0.0)), ID.Puncture(0.3, (1.0, 0.3, 0.0))],
                           seed=1)
    dt = 0.25 * grid.dx
    evo = BSSNEvolution(grid, ko_sigma=0.1, bc=bc, ko_order=ko_order)
    nsteps = 3
    out = evo.evolve(BSSNState(_dev(U)), dt, nsteps, t0=0.2).data.cpu().numpy()
    S = _S(grid.dx, grid.dy, grid.dz, dt=dt, t=0.2)
    ref = U
    for s in range(nsteps):
        S[6] = 0.2 + s * dt if s == 0 else S[6] + dt
        ref = O.rk4_step(ref, S, ko_sigma=0.1, ko_order=ko_order, periodic=(bc == "periodic"), ng=ng)
    assert O.normwise_rel_grouped(out, ref).max() < 1e-12


def test_graph_replay_matches_eager():
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.evolve import BSSNEvolution
    from bssn3d_b200.state import BSSNState
    grid, U, dt = ID.workload(0, n=10)
    evo = BSSNEvolution(grid, ko_sigma=0.1, bc="none", ko_order=6)
    a = evo.evolve(BSSNState(_dev(U)), dt, 2, use_graph=True).data.cpu().numpy()
    b = evo.evolve(BSSNState(_dev(U)), dt, 2, use_graph=False).data.cpu().numpy()
    np.testing.assert_array_equal(a, b)


# ----------------------------------------------------------------- errors
def test_error_paths_do_not_launch():
    L = _lib()
    lib = L.load()
    F = torch.zeros((24, 8, 8, 8), dtype=torch.float64, device=DEV)
    S = torch.zeros(16, dtype=torch.float64, device=DEV)
    out = torch.empty_like(F)
    acc = torch.empty_like(F)
    rc = lib.bssn_b200_rhs(None, F.data_ptr(), S.data_ptr(), out.data_ptr(), 0, 8, 8)
    assert rc == L.EINVAL
    rc = lib.bssn_b200_rhs(None, F.data_ptr(), S.data_ptr(), F.data_ptr(), 8, 8, 8)
    assert rc == L.EINVAL                       # OUT aliases F
    rc = lib.bssn_b200_rk4_stage(None, 5, F.data_ptr(), F.data_ptr(), acc.data_ptr(), out.data_ptr(),
                                 S.data_ptr(), 0.1, 6, 1e-4, 1e-4, 8, 8, 8)
    assert rc == L.EINVAL
    rc = lib.bssn_b200_rk4_stage(None, 0, F.data_ptr(), F.data_ptr(), acc.data_ptr(), F.data_ptr(),
                                 S.data_ptr(), 0.1, 6, 1e-4, 1e-4, 8, 8, 8)
    assert rc == L.EINVAL                       # YNEXT aliases Y
    assert "alias" in lib.bssn_b200_last_error().decode()
    rc = lib.bssn_b200_rk4_stage(None, 0, F.data_ptr(), F.data_ptr(), acc.data_ptr(), out.data_ptr(),
                                 S.data_ptr(), 0.1, 7, 1e-4, 1e-4, 8, 8, 8)
    assert rc == L.EINVAL                       # KO order 7
    torch.cuda.synchronize()


def test_nan_input_propagates_without_fault():
    F = _random_state((12, 12, 12), 3)
    F[5, 6, 6, 6] = np.nan
    out = _gpu_rhs(F, _S(0.1, 0.1, 0.1))
    assert np.isnan(out).any()
    assert np.isfinite(out[:, 0, 0, 0]).all()


# ------------------------------------------------------------ constraints
def test_constraints_golden_and_norms():
    from bssn3d_b200.constraints import ConstraintSolver
    from bssn3d_b200.grid import Grid
    g = np.load(GOLDEN / "bl_small.npz")
    grid = Grid.from_domain(6, lo=-4.0, hi=4.0, ng=3)
    cs = ConstraintSolver(grid)
    out = cs.constraints_tensor(_dev(g["U"])).cpu().numpy()
    assert np.abs(out[0] - g["H"]).max() <= 1e-12 * np.abs(g["H"]).max()
    if np.abs(g["M"]).max() > 0:
        assert np.abs(out[1:] - g["M"]).max() <= 1e-12 * np.abs(g["M"]).max()
    h, m = cs.l2(_dev(g["U"]))
    sl = (slice(3, -3),) * 3
    assert h == pytest.approx(float(np.sqrt(np.mean(g["H"][sl] ** 2))), rel=1e-12)


def test_constraints_random_vs_oracle():
    from bssn3d_b200.constraints import ConstraintSolver
    from bssn3d_b200.grid import Grid
    F = _random_state((19, 21, 23), 8)
    grid = Grid(Nx=13, Ny=15, Nz=17, dx=0.1, dy=0.11, dz=0.09, ng=3)
    out = ConstraintSolver(grid).constraints_tensor(_dev(F)).cpu().numpy()
    H, M = O.constraints(F, 0.1, 0.11, 0.09)
    assert O.normwise_rel(out, np.concatenate([H[None], M])).max() < 1e-12


def test_constraint_norms_fused_vs_oracle_and_reproducible():
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.constraints import ConstraintSolver
    grid, U, _ = ID.workload(0, n=20)
    cs = ConstraintSolver(grid)
    a = cs.l2_tensor(_dev(U)).cpu().numpy()
    b = cs.l2_tensor(_dev(U)).cpu().numpy()
    np.testing.assert_array_equal(a, b)                     # fixed-order reduction
    h, m = O.constraint_norms(U, grid.dx, grid.dy, grid.dz, grid.ng)
    assert a[0] == pytest.approx(h, rel=1e-12)
    assert a[1] == pytest.approx(m, rel=1e-12, abs=1e-300)


def _reference_vector_recipe(npts=1 << 18, seed=1):
    """Inputs of the reference's algebra-only vector file
    (3D/src/bssn3d/cuda/gen_algebra_cuda.py:99-140): near-Minkowski fields
    (1 or 0 plus 0.03 N(0,1), drawn in state order), derivatives 0.03 N(0,1),
    default physics, dt 0.01, dx 0.1, t 0."""
    rng = np.random.default_rng(seed)
    F = np.empty((24, npts))
    for f in range(24):
        F[f] = (1.0 if f in (0, 1, 3, 6, 8) else 0.0) + 0.03 * rng.standard_normal(npts)
    D = 0.03 * rng.standard_normal((138, npts))
    S = _S(0.1, 0.1, 0.1, dt=0.01, t=0.0)
    return F, D, S


def test_algebra_reference_vector_recipe():
    F, D, S = _reference_vector_recipe()
    Fd, Dd, Sd = _dev(F), _dev(D), _dev(S)
    out = torch.empty_like(Fd)
    L = _lib()
    L.check(L.load().bssn_b200_rhs_algebra(None, Fd.data_ptr(), Dd.data_ptr(), Sd.data_ptr(), out.data_ptr(),
                                           F.shape[1]))
    got = out.cpu().numpy()
    assert np.isfinite(got).all()
    assert O.normwise_rel(got, O.rhs_algebra(F, D, S)).max() < 1e-12
    if O.have_ref():
        assert O.normwise_rel(got, O.ref_rhs_algebra(F, D, S)).max() < 1e-12
