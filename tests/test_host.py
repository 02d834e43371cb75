"""Host-side logic that needs no GPU: the C-ABI library loads and exports
every symbol include/bssn_b200.h declares, the scalar pack and field orders
match the reference's boundary, argument validation, initial data.

Mirrors the CPU-checkable invariants of
3D/tests/integration/test_bssn_fused_cuda.py:20-38 (scalar packing, output
order, missing-library error).
"""

import re
from pathlib import Path

import numpy as np
import pytest

from conftest import ROOT
from bssn3d_b200 import _lib
from bssn3d_b200 import initial_data as ID
from bssn3d_b200.fused_rhs import pack_S, NSCAL
from bssn3d_b200.grid import Grid
from bssn3d_b200.state import VAR_NAMES, OUTPUT_FIELDS, FIELD_INPUTS, PhysicsParams


def _declared_symbols():
    text = (ROOT / "include" / "bssn_b200.h").read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(bssn_b200_\w+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = _lib.load()
    declared = _declared_symbols()
    assert declared, "no declarations parsed"
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(_lib.exported_symbols()) == declared
    assert lib.bssn_b200_version().decode().startswith("bssn_b200")


def test_pack_order_matches_reference_boundary():
    S = pack_S(1.0, 2.0, 3.0, 4.0, 5.0, 6.0, 7.0, (8.0, 9.0, 10.0, 11.0), (12.0, 13.0), 14.0, 15.0)
    assert S.shape == (NSCAL,)
    np.testing.assert_array_equal(S, [1, 2, 3, 4, 5, 6, 7, 8, 9, 10, 11, 12, 13, 4, 14, 15])


def test_field_orders():
    assert FIELD_INPUTS == VAR_NAMES == OUTPUT_FIELDS
    assert VAR_NAMES[:3] == ["alpha", "chi", "K"] and VAR_NAMES[-1] == "B2"
    assert len(VAR_NAMES) == 24


def test_missing_library_raises(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "LIB_PATH", tmp_path / "absent.so")
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(FileNotFoundError, match="build"):
        _lib.load()


def test_solver_validation():
    from bssn3d_b200.rhs import BSSNSolver
    g3 = Grid.from_domain(16, ng=3)
    with pytest.raises(ValueError, match="ng>="):
        BSSNSolver(g3, order=6, ko_order=8)      # KO8 needs 4 ghosts (rhs.py:92-96)
    BSSNSolver(g3, order=6, ko_order=6)
    with pytest.raises(ValueError):
        BSSNSolver(g3, order=6, ko_order=6, scheme="verbatim")
    with pytest.raises(ValueError):
        BSSNSolver(g3, order=4, ko_order=6)
    s = BSSNSolver(g3, order=6, ko_order=6)
    assert s.dt == pytest.approx(0.25 * g3.dx)


def test_grid_matches_reference_layout():
    g = Grid.from_domain(64, lo=-4.0, hi=4.0, ng=3)
    assert g.shape == (70, 70, 70)
    assert g.dx == 0.125
    assert g.x[0] == -4.0 - 3 * 0.125
    assert np.isclose(g.x[3 + 64 - 1], 4.0 - 0.125)
    assert Grid.from_domain(8).ng == 4


def test_brill_lindquist_data():
    grid, U, dt = ID.workload(0, n=8)
    assert U.shape == (24, 14, 14, 14)
    g = U[3:9]
    det = g[0] * (g[3] * g[5] - g[4] ** 2) - g[1] * (g[1] * g[5] - g[4] * g[2]) + g[2] * (g[1] * g[4] - g[3] * g[2])
    np.testing.assert_allclose(det, 1.0, atol=1e-15)
    np.testing.assert_allclose(U[1], U[0] ** 2, rtol=1e-14)       # chi = psi^-4 = alpha^2
    assert np.all(U[9:12] == 0) and np.all(U[12:24] == 0) and np.all(U[2] == 0)
    assert dt == 0.25 * grid.dx
    # seeded: the same call gives the same bytes
    _, U2, _ = ID.workload(0, n=8)
    np.testing.assert_array_equal(U, U2)
    # with dx = 0.5 the punctures at x = +-1.5 sit on nodes: r is floored at dx/2
    grid, U, _ = ID.workload(0, n=16)
    psi = 1.0 + 0.5 / (2 * 0.25) + 0.5 / (2 * 3.0)
    assert np.isclose(U[1].min(), psi ** -4, rtol=1e-12)


def test_physics_defaults():
    p = PhysicsParams()
    assert (p.eta, p.lmbda, p.lambda_f, p.cahd_c, p.ssl_h, p.ssl_sigma) == \
        (2.0, (1.0, 1.0, 1.0, 1.0), (1.0, 0.0), 0.06, 0.6, 20.0)
