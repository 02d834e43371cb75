"""ctypes binding of the C ABI in include/bssn_b200.h.

The library is mandatory: there is no CPU or PyTorch fallback. If
``libbssn_b200.so`` is missing the import of any compute entry point raises
``FileNotFoundError`` naming the build step, like the reference's
``fused_rhs_cuda._register`` (3D/src/bssn3d/fused_rhs_cuda.py:41-49).
"""

from __future__ import annotations

import ctypes
from pathlib import Path

LIB_PATH = Path(__file__).resolve().parent / "libbssn_b200.so"
HEADER = Path(__file__).resolve().parents[2] / "include" / "bssn_b200.h"

OK, EINVAL, ECUDA = 0, 1, 3
NVARIANTS = 4  # BSSN_B200_NVARIANTS

_P = ctypes.c_void_p
_LL = ctypes.c_longlong
_D = ctypes.c_double
_I = ctypes.c_int
_SZ = ctypes.c_size_t

_SIGNATURES = {
    "bssn_b200_last_error": ([], ctypes.c_char_p),
    "bssn_b200_version": ([], ctypes.c_char_p),
    "bssn_b200_async_copy_errors": ([_P], _I),
    "bssn_b200_rhs": ([_P, _P, _P, _P, _LL, _LL, _LL], _I),
    "bssn_b200_constraints": ([_P, _P, _P, _P, _LL, _LL, _LL], _I),
    "bssn_b200_norms_scratch_bytes": ([], _SZ),
    "bssn_b200_constraint_norms": ([_P, _P, _P, _LL, _LL, _LL, _I, _P, _SZ, _P], _I),
    "bssn_b200_constraint_norms_static": ([_P, _P, _P, _LL, _LL, _LL, _I, _P], _I),
    "bssn_b200_batch_plan": ([_P, _I, _I], _I),
    "bssn_b200_fill_plan": ([_P, _I, _LL], _LL),
    "bssn_b200_fill": ([_P, _P, _P, _I, _LL, _P], _I),
    "bssn_b200_batch_rhs": ([_P, _P, _P, _P, _P, _I, _I, _I], _I),
    "bssn_b200_batch_rk4_stage": ([_P, _I, _P, _P, _P, _P, _P, _D, _I, _D, _D, _P, _I, _I, _I], _I),
    "bssn_b200_rk4_stage": ([_P, _I, _P, _P, _P, _P, _P, _D, _I, _D, _D, _LL, _LL, _LL], _I),
    "bssn_b200_msrk_stage": ([_P, _I, _P, _P, _P, _P, _P, _P, _P, _P, _D, _I, _D, _D, _LL, _LL, _LL], _I),
    "bssn_b200_derivatives": ([_P, _P, _P, _P, _D, _I, _LL, _LL, _LL], _I),
    "bssn_b200_advance_time": ([_P, _P], _I),
    "bssn_b200_rhs_algebra": ([_P, _P, _P, _P, _P, _LL], _I),
    "bssn_b200_ozaki_workspace_bytes": ([_LL, _LL, _LL, _I], _SZ),
    "bssn_b200_ozaki_error_flag": ([_P, _LL, _LL, _LL, _I], _P),
    "bssn_b200_ozaki_last_error": ([], ctypes.c_char_p),
    "bssn_b200_ozaki_derivatives": ([_P, _P, _P, _P, _I, _D, _I, _LL, _LL, _LL, _P, _SZ], _I),
    "bssn_b200_batch_ozaki_plan": ([_P, _I, _P, _P, _P], _LL),
    "bssn_b200_batch_ozaki_derivatives": ([_P, _P, _P, _P, _I, _D, _I, _P, _I, _P, _P, _P, _SZ], _I),
    "bssn_b200_batch_rk4_stage_derivs": ([_P, _I, _P, _P, _P, _P, _P, _P, _I, _D, _D, _P, _I, _P, _LL], _I),
    "bssn_b200_enforce": ([_P, _P, _LL, _D, _D], _I),
    "bssn_b200_periodic_sync": ([_P, _P, _LL, _LL, _LL, _I], _I),
}

_lib = None


class BssnB200Error(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"bssn_b200 status {code}: {msg}")
        self.code = code


def load() -> ctypes.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not LIB_PATH.exists():
        raise FileNotFoundError(
            f"{LIB_PATH} not built. Build it with: python integer-schemes_b200/build.py")
    lib = ctypes.CDLL(str(LIB_PATH))
    for name, (args, res) in _SIGNATURES.items():
        fn = getattr(lib, name)
        fn.argtypes = args
        fn.restype = res
    _lib = lib
    return lib


def check(rc: int) -> None:
    if rc != OK:
        msg = load().bssn_b200_last_error().decode(errors="replace")
        raise BssnB200Error(rc, msg)


def exported_symbols():
    return list(_SIGNATURES)
