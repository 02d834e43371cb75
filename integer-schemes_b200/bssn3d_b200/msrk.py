"""Coefficients of the 2-step / 3-stage multistep Runge-Kutta methods that
``BSSNEvolution(integrator=...)`` accepts, and their linear stability.

The methods are RK4-2(1) and RK4-2(2) of Sanches, Brandt, Kalinani, Ji &
Schnetter, "Accelerating Numerical Relativity Simulations with New Multistep
Fourth-Order Runge-Kutta Methods" (arXiv:2603.05763), Table 1 — the same
tables the reference carries in 2D/src/mcs2d/msrk.py:38-56 and selects in
3D/src/bssn3d/evolve.py:42-55. A step reuses the previous step's
f(y_{n-1}) as its stage 0, so it makes 3 fresh RHS evaluations instead of 4:

    k0 = f(y_{n-1}),  k1 = f(y_n, t)
    Y2 = y_n + dt (a20 k0 + a21 k1),              k2 = f(Y2, t + c2 dt)
    Y3 = y_n + dt (a30 k0 + a31 k1 + a32 k2),     k3 = f(Y3, t + c3 dt)
    y_{n+1} = enforce(y_n + dt (b0 k0 + b1 k1 + b2 k2 + b3 k3))

with c2 = a20 + a21 and c3 = a30 + a31 + a32. ``coef`` packs
(a20, a21, a30, a31, a32, b0, b1, b2, b3) in the order the C ABI's
``bssn_b200_msrk_stage`` takes them.

The stability helpers apply the step to the model problem y' = lambda y
(z = lambda dt) and bound the spectral radius of the 2x2 recurrence matrix;
the imaginary-axis intercept they give is checked against the paper's
published values (RK4 sqrt(8); RK4-2(1) 2.53865; RK4-2(2) 2.46201).
"""

from __future__ import annotations

from dataclasses import dataclass
from fractions import Fraction as Fr
from typing import Dict, Tuple

import numpy as np


@dataclass(frozen=True)
class Method:
    name: str
    a20: Fr
    a21: Fr
    a30: Fr
    a31: Fr
    a32: Fr
    b: Tuple[Fr, Fr, Fr, Fr]
    c2: Fr
    c3: Fr

    def check(self) -> None:
        """Consistency conditions in exact arithmetic: sum(b) = 1 and the
        nodes are the row sums of the stage matrix."""
        if sum(self.b) != 1:
            raise ValueError(f"{self.name}: sum(b) != 1")
        if self.a20 + self.a21 != self.c2 or self.a30 + self.a31 + self.a32 != self.c3:
            raise ValueError(f"{self.name}: node is not the row sum")

    @property
    def coef(self) -> Tuple[float, ...]:
        return tuple(float(v) for v in (self.a20, self.a21, self.a30, self.a31, self.a32, *self.b))

    def recurrence(self, z: complex) -> np.ndarray:
        """M(z) with (y_{n+1}, y_n) = M(z) (y_n, y_{n-1}) for y' = lambda y."""
        a20, a21, a30, a31, a32 = (float(v) for v in (self.a20, self.a21, self.a30, self.a31, self.a32))
        b0, b1, b2, b3 = (float(v) for v in self.b)

        def advance(yn: complex, yprev: complex) -> complex:
            g0, g1 = z * yprev, z * yn
            g2 = z * (yn + a20 * g0 + a21 * g1)
            g3 = z * (yn + a30 * g0 + a31 * g1 + a32 * g2)
            return yn + b0 * g0 + b1 * g1 + b2 * g2 + b3 * g3

        return np.array([[advance(1.0, 0.0), advance(0.0, 1.0)], [1.0, 0.0]], dtype=np.complex128)


METHODS: Dict[str, Method] = {
    "rk4_2_1": Method("rk4_2_1",
                      a20=Fr(-49, 1250), a21=Fr(399, 1250),
                      a30=Fr(7033, 960000), a31=Fr(-217633, 210000), a32=Fr(5473, 10752),
                      b=(Fr(-643, 1536), Fr(-4237, 1092), Fr(38125, 10752), Fr(4375, 2496)),
                      c2=Fr(7, 25), c3=Fr(-13, 25)),
    "rk4_2_2": Method("rk4_2_2",
                      a20=Fr(1309, 15500), a21=Fr(-31999, 15500),
                      a30=Fr(-241289, 5880000), a31=Fr(22846301, 16170000), a32=Fr(-936169, 2587200),
                      b=(Fr(-191, 882), Fr(48241, 59994), Fr(193750, 4351347), Fr(100000, 271791)),
                      c2=Fr(-99, 50), c3=Fr(101, 100)),
}
for _m in METHODS.values():
    _m.check()

# fresh RHS evaluations per step
STAGES = {"rk4": 4, "rk4_2_1": 3, "rk4_2_2": 3}


def spectral_radius(z: complex, method: str) -> float:
    if method == "rk4":
        return float(abs(1 + z + z ** 2 / 2 + z ** 3 / 6 + z ** 4 / 24))
    return float(np.max(np.abs(np.linalg.eigvals(METHODS[method].recurrence(z)))))


def imag_axis_intercept(method: str, tol: float = 1e-7) -> float:
    """Largest B such that i*beta is in the absolute-stability region for the
    whole segment 0 < beta <= B (root condition with a 1e-9 slack).

    A scan at step 1e-3 finds the first unstable beta, then bisection
    narrows the crossing to ``tol``."""
    def stable(beta: float) -> bool:
        return spectral_radius(1j * beta, method) <= 1.0 + 1e-9

    step = 1e-3
    beta = step
    while stable(beta):
        beta += step
        if beta > 64.0:
            return float("inf")
    lo, hi = beta - step, beta
    while hi - lo > tol:
        mid = 0.5 * (lo + hi)
        lo, hi = (mid, hi) if stable(mid) else (lo, mid)
    return 0.5 * (lo + hi)


def get(name: str) -> Method:
    """The method for an ``integrator`` name; raises like evolve.py:50-55."""
    if name not in METHODS:
        raise ValueError(f"integrator {name!r}: only 'rk4' or a 2-step rk4_2_* MSRK method "
                         f"are supported here")
    return METHODS[name]
