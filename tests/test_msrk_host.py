"""MSRK method tables and their linear stability (no GPU).

The imaginary-axis intercepts pin the transcribed coefficient tables against
the values the paper publishes (2D/tests/integration/test_msrk.py:21-31); the
oracle's MSRK step is checked against its own RK4 step for 4th-order
agreement on a small gauge wave."""

import numpy as np
import pytest
from fractions import Fraction

from bssn3d_b200 import msrk

PAPER_INTERCEPT = {"rk4": np.sqrt(8.0), "rk4_2_1": 2.53865, "rk4_2_2": 2.46201}


@pytest.mark.parametrize("method", ["rk4", "rk4_2_1", "rk4_2_2"])
def test_imag_axis_intercept_matches_paper(method):
    assert abs(msrk.imag_axis_intercept(method) - PAPER_INTERCEPT[method]) < 1e-4


def test_coefficients_consistent_and_packed_in_abi_order():
    for name, m in msrk.METHODS.items():
        assert sum(m.b) == 1
        assert m.a20 + m.a21 == m.c2 and m.a30 + m.a31 + m.a32 == m.c3
        c = m.coef
        assert len(c) == 9 and all(isinstance(v, float) for v in c)
        assert c[:5] == tuple(float(v) for v in (m.a20, m.a21, m.a30, m.a31, m.a32))
        assert c[5:] == tuple(float(v) for v in m.b)
        assert abs(sum(c[5:]) - 1.0) < 1e-15
    assert msrk.STAGES == {"rk4": 4, "rk4_2_1": 3, "rk4_2_2": 3}


def test_inconsistent_table_is_rejected():
    m = msrk.METHODS["rk4_2_2"]
    bad = msrk.Method("bad", m.a20, m.a21, m.a30, m.a31, m.a32,
                      (m.b[0] + Fraction(1, 10**6),) + m.b[1:], m.c2, m.c3)
    with pytest.raises(ValueError):
        bad.check()


@pytest.mark.parametrize("name", ["rk4_3", "msrk", "rk3"])
def test_unsupported_integrators_raise(name):
    with pytest.raises(ValueError, match="2-step"):
        msrk.get(name)


def test_scalar_problem_is_fourth_order():
    """y' = lambda y over a fixed time: the global error of the MSRK recurrence
    (RK4 start) falls ~16x per halving of dt."""
    lam = -1.0 + 2.0j
    T = 1.0

    def run(method, n):
        dt = T / n
        z = lam * dt
        y1 = 1 + z + z ** 2 / 2 + z ** 3 / 6 + z ** 4 / 24   # RK4 start
        M = msrk.METHODS[method].recurrence(z)
        v = np.array([y1, 1.0], dtype=np.complex128)
        for _ in range(n - 1):
            v = M @ v
        return abs(v[0] - np.exp(lam * T))

    for method in msrk.METHODS:
        e1, e2 = run(method, 64), run(method, 128)
        assert 3.7 < np.log2(e1 / e2) < 4.3


def test_oracle_msrk_agrees_with_oracle_rk4_to_truncation():
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.grid import Grid
    from bssn3d_b200.fused_rhs import pack_S
    from oracle import oracle as O
    g = Grid.from_domain(10, ko_order=6)
    U = ID.gauge_wave(g, amplitude=0.01)
    dt = 0.1 * g.dx
    S = pack_S(2.0, 0.06, dt, g.dx, 0.6, 20.0, 0.0, (1, 1, 1, 1), (1, 0), g.dy, g.dz)
    y4 = U
    S4 = S.copy()
    for _ in range(6):
        y4 = O.rk4_step(y4, S4, ko_sigma=0.4, ko_order=6, periodic=True, ng=g.ng)
        S4[6] += dt
    y2 = O.msrk_evolve(U, S, msrk.METHODS["rk4_2_2"].coef, 6, ko_sigma=0.4, ko_order=6,
                       periodic=True, ng=g.ng)
    assert np.isfinite(y2).all()
    rms = lambda a: float(np.sqrt(np.mean(a ** 2)))
    assert rms(y2 - y4) / rms(y4) < 1e-6
