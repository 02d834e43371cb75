"""TEST INFRASTRUCTURE — ctypes front end of the CPU oracle.

Only tests/, ``__graft_entry__.smoke()`` and bench.py's CPU-baseline leg import
this module, and only as the checker. It loads

* ``oracle/liboracle.so`` — the plain-C restatement of the reference path
  (``oracle/bssn_oracle.c``), and
* ``oracle/_ref/libdendro_ref.so`` — the reference's own Dendro-GR algebra
  (``3D/src/bssn3d/vendor/bssneqs_SSL_HD_dxsq.cpp``) compiled where it lies by
  ``oracle/Makefile``; present only where it was built.

Array conventions follow the C-ABI: fields ``(24, Sx, Sy, Sz)`` float64 in
state order (``3D/src/bssn3d/state.py:37-46``), derivatives ``(138, ...)``,
the 16-scalar pack of ``3D/src/bssn3d/fused_rhs_cuda.py:52-55``.
"""

from __future__ import annotations

import ctypes
import os
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB_PATH = HERE / "liboracle.so"
REF_PATH = HERE / "_ref" / "libdendro_ref.so"

_P = ctypes.POINTER(ctypes.c_double)
_L = ctypes.c_long
_D = ctypes.c_double
_I = ctypes.c_int

_lib = None
_ref = None


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(_P)


def _c(a) -> np.ndarray:
    return np.ascontiguousarray(a, dtype=np.float64)


def lib():
    """The restatement library (built by ``make -C oracle``)."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise FileNotFoundError(f"{LIB_PATH} not built: run `make -C oracle`")
        L = ctypes.CDLL(str(LIB_PATH))
        L.oracle_derivatives.argtypes = [_P, _L, _L, _L, _D, _D, _D, _P]
        L.oracle_ko.argtypes = [_P, _L, _L, _L, _D, _D, _D, _D, _I, _P]
        L.oracle_rhs_algebra.argtypes = [_L, _P, _P, _P, _P, _P]
        L.oracle_rhs.argtypes = [_P, _L, _L, _L, _P, _P]
        L.oracle_hamiltonian.argtypes = [_P, _L, _L, _L, _D, _D, _D, _P]
        L.oracle_enforce.argtypes = [_P, _L, _D, _D]
        L.oracle_constraints.argtypes = [_P, _L, _L, _L, _D, _D, _D, _P, _P]
        L.oracle_constraints_algebra.argtypes = [_L, _P, _P, _P, _P]
        L.oracle_periodic_sync.argtypes = [_P, _L, _L, _L, _I]
        L.oracle_rk4_step.argtypes = [_P, _L, _L, _L, _P, _D, _I, _I, _I, _D, _D, _P]
        L.oracle_rate.argtypes = [_P, _L, _L, _L, _P, _D, _I, _I, _I, _P]
        L.oracle_msrk2_step.argtypes = [_P, _P, _L, _L, _L, _P, _P, _D, _I, _I, _I, _D, _D, _P, _P]
        _lib = L
    return _lib


PHYSCON_PATH = HERE / "_ref" / "libdendro_physcon.so"
_physcon = None


def have_ref() -> bool:
    return REF_PATH.exists()


def have_physcon() -> bool:
    return PHYSCON_PATH.exists()


def physcon_lib():
    """The reference's compiled constraint block (``oracle/_ref``)."""
    global _physcon
    if _physcon is None:
        if not PHYSCON_PATH.exists():
            raise FileNotFoundError(f"{PHYSCON_PATH} not built: run `make -C oracle ref`")
        L = ctypes.CDLL(str(PHYSCON_PATH))
        L.dendro_ref_constraints.argtypes = [_L, _P, _P, _P, _P, _I]
        L.dendro_ref_constraints.restype = _I
        _physcon = L
    return _physcon


def ref_lib():
    """The reference's compiled algebra (``oracle/_ref``)."""
    global _ref
    if _ref is None:
        if not REF_PATH.exists():
            raise FileNotFoundError(f"{REF_PATH} not built: run `make -C oracle ref`")
        L = ctypes.CDLL(str(REF_PATH))
        L.dendro_ref_rhs_algebra.argtypes = [_L, _P, _P, _P, _P, _I]
        L.dendro_ref_rhs_algebra.restype = _I
        _ref = L
    return _ref


# ---------------------------------------------------------------------------

def derivatives(F: np.ndarray, dx: float, dy: float, dz: float) -> np.ndarray:
    F = _c(F)
    _, Sx, Sy, Sz = F.shape
    D = np.empty((138, Sx, Sy, Sz))
    lib().oracle_derivatives(_ptr(F), Sx, Sy, Sz, dx, dy, dz, _ptr(D))
    return D


def ko(F: np.ndarray, dx, dy, dz, sigma: float, ko_order: int = 6) -> np.ndarray:
    F = _c(F)
    _, Sx, Sy, Sz = F.shape
    out = np.empty_like(F)
    lib().oracle_ko(_ptr(F), Sx, Sy, Sz, dx, dy, dz, sigma, ko_order, _ptr(out))
    return out


def rhs_algebra(F: np.ndarray, D: np.ndarray, S: np.ndarray, want_H: bool = False):
    """Pointwise algebra; F (24, n...) and D (138, n...) with matching tails."""
    F = _c(F)
    D = _c(D)
    S = _c(S)
    n = int(np.prod(F.shape[1:]))
    out = np.empty_like(F)
    H = np.empty(F.shape[1:]) if want_H else None
    lib().oracle_rhs_algebra(n, _ptr(F), _ptr(D), _ptr(S), _ptr(out),
                             _ptr(H) if want_H else None)
    return (out, H) if want_H else out


def ref_rhs_algebra(F: np.ndarray, D: np.ndarray, S: np.ndarray, nthreads: int = 1):
    """The reference's compiled algebra on the same inputs."""
    F = _c(F)
    D = _c(D)
    S = _c(S)
    n = int(np.prod(F.shape[1:]))
    out = np.empty_like(F)
    ref_lib().dendro_ref_rhs_algebra(n, _ptr(F), _ptr(D), _ptr(S), _ptr(out), nthreads)
    return out


def rhs(F: np.ndarray, S: np.ndarray) -> np.ndarray:
    """Full RHS of a state: restated stencils + restated algebra."""
    F = _c(F)
    S = _c(S)
    _, Sx, Sy, Sz = F.shape
    out = np.empty_like(F)
    lib().oracle_rhs(_ptr(F), Sx, Sy, Sz, _ptr(S), _ptr(out))
    return out


def ref_rhs(F: np.ndarray, S: np.ndarray, nthreads: int = 1) -> np.ndarray:
    """Full RHS with the reference's own compiled algebra."""
    D = derivatives(F, S[13], S[14], S[15])
    return ref_rhs_algebra(F, D, S, nthreads)


def hamiltonian(F: np.ndarray, dx, dy, dz) -> np.ndarray:
    F = _c(F)
    _, Sx, Sy, Sz = F.shape
    H = np.empty((Sx, Sy, Sz))
    lib().oracle_hamiltonian(_ptr(F), Sx, Sy, Sz, dx, dy, dz, _ptr(H))
    return H


def constraints(F: np.ndarray, dx, dy, dz):
    """(H, M) fields of a state: H (Sx,Sy,Sz), M (3,Sx,Sy,Sz)."""
    F = _c(F)
    _, Sx, Sy, Sz = F.shape
    H = np.empty((Sx, Sy, Sz))
    M = np.empty((3, Sx, Sy, Sz))
    lib().oracle_constraints(_ptr(F), Sx, Sy, Sz, dx, dy, dz, _ptr(H), _ptr(M))
    return H, M


def constraints_algebra(F: np.ndarray, D: np.ndarray):
    F = _c(F)
    D = _c(D)
    n = int(np.prod(F.shape[1:]))
    H = np.empty(F.shape[1:])
    M = np.empty((3,) + F.shape[1:])
    lib().oracle_constraints_algebra(n, _ptr(F), _ptr(D), _ptr(H), _ptr(M))
    return H, M


def ref_constraints_algebra(F: np.ndarray, D: np.ndarray, nthreads: int = 1):
    """The reference's compiled constraints on the same inputs."""
    F = _c(F)
    D = _c(D)
    n = int(np.prod(F.shape[1:]))
    H = np.empty(F.shape[1:])
    M = np.empty((3,) + F.shape[1:])
    physcon_lib().dendro_ref_constraints(n, _ptr(F), _ptr(D), _ptr(H), _ptr(M), nthreads)
    return H, M


def constraint_norms(F: np.ndarray, dx, dy, dz, ng: int):
    """Interior L2 norms (H, |M|) of 3D/src/bssn3d/constraints.py:53-62."""
    H, M = constraints(F, dx, dy, dz)
    sl = (slice(ng, -ng),) * 3
    h = H[sl]
    m = M[(slice(None),) + sl]
    return float(np.sqrt(np.mean(h ** 2))), float(np.sqrt(np.mean((m ** 2).sum(axis=0))))


def enforce(F: np.ndarray, chi_floor=1e-4, alpha_floor=1e-4) -> np.ndarray:
    F = _c(F).copy()
    n = int(np.prod(F.shape[1:]))
    lib().oracle_enforce(_ptr(F), n, chi_floor, alpha_floor)
    return F


def periodic_sync(F: np.ndarray, ng: int) -> np.ndarray:
    F = _c(F).copy()
    _, Sx, Sy, Sz = F.shape
    lib().oracle_periodic_sync(_ptr(F), Sx, Sy, Sz, ng)
    return F


def rk4_step(F: np.ndarray, S: np.ndarray, ko_sigma=0.1, ko_order=6,
             periodic=False, ng=3, chi_floor=1e-4, alpha_floor=1e-4) -> np.ndarray:
    """One RK4 step + enforce. ``S[2]`` is dt, ``S[6]`` the step's start time."""
    F = _c(F)
    S = _c(S)
    _, Sx, Sy, Sz = F.shape
    out = np.empty_like(F)
    lib().oracle_rk4_step(_ptr(F), Sx, Sy, Sz, _ptr(S), ko_sigma, ko_order,
                          int(periodic), ng, chi_floor, alpha_floor, _ptr(out))
    return out


def rate(F: np.ndarray, S: np.ndarray, ko_sigma=0.1, ko_order=6, periodic=False, ng=3) -> np.ndarray:
    """RHS + KO at time S[6] (BSSNEvolution.rhs, evolve.py:86-91)."""
    F = _c(F)
    S = _c(S)
    _, Sx, Sy, Sz = F.shape
    out = np.empty_like(F)
    lib().oracle_rate(_ptr(F), Sx, Sy, Sz, _ptr(S), ko_sigma, ko_order, int(periodic), ng, _ptr(out))
    return out


def msrk2_step(F: np.ndarray, fprev: np.ndarray, S: np.ndarray, coef, ko_sigma=0.1, ko_order=6,
               periodic=False, ng=3, chi_floor=1e-4, alpha_floor=1e-4):
    """One 2-step / 3-stage MSRK step + enforce (evolve.py:139-153).
    coef = (a20, a21, a30, a31, a32, b0, b1, b2, b3). Returns (y_{n+1}, f(y_n))."""
    F = _c(F)
    K = _c(fprev)
    S = _c(S)
    c = _c(np.asarray(coef, dtype=np.float64))
    _, Sx, Sy, Sz = F.shape
    out = np.empty_like(F)
    kout = np.empty_like(F)
    lib().oracle_msrk2_step(_ptr(F), _ptr(K), Sx, Sy, Sz, _ptr(S), _ptr(c), ko_sigma, ko_order,
                            int(periodic), ng, chi_floor, alpha_floor, _ptr(out), _ptr(kout))
    return out, kout


def msrk_evolve(F: np.ndarray, S: np.ndarray, coef, nsteps: int, ko_sigma=0.1, ko_order=6,
                periodic=False, ng=3) -> np.ndarray:
    """BSSNEvolution.evolve with an MSRK integrator (evolve.py:167-183):
    f0 = rate(y0), one RK4 step, then nsteps-1 MSRK steps. S[6] is t0."""
    S = _c(S).copy()
    dt = S[2]
    f = rate(F, S, ko_sigma, ko_order, periodic, ng)
    y = rk4_step(F, S, ko_sigma, ko_order, periodic, ng)
    for _ in range(1, int(nsteps)):
        S[6] = S[6] + dt
        y, f = msrk2_step(y, f, S, coef, ko_sigma, ko_order, periodic, ng)
    return y


def normwise_rel(a: np.ndarray, b: np.ndarray, floor: float = 1e-300) -> np.ndarray:
    """Per-field max|a-b| / max(max|b|, floor); fields along axis 0."""
    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    num = np.max(np.abs(a - b), axis=1)
    den = np.maximum(np.max(np.abs(b), axis=1), floor)
    return np.where(num == 0.0, 0.0, num / den)


# tensor groups of the state: alpha, chi, K, gt (6), beta (3), At (6), Gt (3), B (3)
GROUPS = [[0], [1], [2], list(range(3, 9)), list(range(9, 12)), list(range(12, 18)),
          list(range(18, 21)), list(range(21, 24))]


def normwise_rel_grouped(a: np.ndarray, b: np.ndarray, floor: float = 1e-300) -> np.ndarray:
    """Per-field max|a-b| divided by the largest |b| over the field's tensor
    (its 1, 3 or 6 components): a component that is pure seeded noise (an
    off-diagonal metric entry of 1e-8) is measured against its tensor's size."""
    a = a.reshape(a.shape[0], -1)
    b = b.reshape(b.shape[0], -1)
    num = np.max(np.abs(a - b), axis=1)
    fmax = np.max(np.abs(b), axis=1)
    den = np.empty_like(fmax)
    for g in GROUPS:
        den[g] = max(float(fmax[g].max()), floor)
    return np.where(num == 0.0, 0.0, num / den)


def set_threads(n: int) -> None:
    os.environ["OMP_NUM_THREADS"] = str(n)
