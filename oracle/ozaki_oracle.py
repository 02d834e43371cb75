"""TEST INFRASTRUCTURE — CPU oracle of the Ozaki INT8 derivative bundle.

Only tests/ import this module, and only as the checker of the tensor-core
passes (``bssn_b200_ozaki_derivatives``, ``bssn_b200_batch_ozaki_derivatives``).

It restates, with numpy integer and float64 arithmetic, what one pass
computes, so that the GPU result can be compared bit for bit:

* the pass covers the box [m, s - m) of the array on each axis,
  m = max(core - ext, 0); lines run along the axis, outputs are grouped in
  16s from the box start;
* the window of a line and output group is its 16 outputs plus R points on
  each side (R = 4 with KO8, else 3), positions clamped to the array (the
  edge padding of derivatives.py:83-84);
* one exponent per window, e = frexp(max |f|)[1] + 1 (0 for an all-zero
  window), so that |f| 2^-e < 1/2;
* X = rint(f 2^-e 2^(7k)) as an int64; digit planes q_0 = X >> 7(k-1)
  (signed) and q_s = (X >> 7(k-1-s)) & 127;
* per plane the exact integer stencil sums C1, C2 (as 2·128 + 14 / −4·128 + 22
  high and low digits) and KO6/KO8 (the banded integer design of the
  reference's MCS Ozaki derivative, 2D/src/mcs2d/schemes/ozaki.py:286-323);
* recombination in float64, planes in pairs from the smallest,
  r += (acc_{s-1}·128 + acc_s) · 2^(-7(s+1)) (exact integer pairs and
  products, one rounding per add; an odd top plane alone), then (r · 2^e) · w with
  w = (1/60)(1/h), (1/180)(1/h²), (1/64 or 1/256)(σ/h);
* the bundle runs the passes of derivative_bundle.py:31-48 — per field the
  x, y, z passes (KO summed x, then y, then z), then the mixed second
  derivatives as the y and z derivatives of the x first derivative and the z
  derivative of the y first derivative.
"""

from __future__ import annotations

import math

import numpy as np

NO = 16
C1 = np.array([-1, 9, -45, 0, 45, -9, 1], dtype=np.int64)
C2H = np.array([0, 0, 2, -4, 2, 0, 0], dtype=np.int64)
C2L = np.array([2, -27, 14, 22, 14, -27, 2], dtype=np.int64)
K6 = np.array([1, -6, 15, -20, 15, -6, 1], dtype=np.int64)
K8 = np.array([-1, 8, -28, 56, -70, 56, -28, 8, -1], dtype=np.int64)

# fields with second derivatives and their slot groups (the slot layout of
# the 138-derivative bundle: d1 at 3f + axis, d2 at 72 + 6 g + pair)
D2_FIELDS = [0, 1] + list(range(3, 12))
PAIR = {(0, 0): 0, (0, 1): 1, (0, 2): 2, (1, 1): 3, (1, 2): 4, (2, 2): 5}
# pass kinds: (axis, halo extension per axis)
KINDS = [(0, (0, 3, 3)), (0, (0, 0, 0)), (1, (0, 0, 3)), (1, (0, 0, 0)), (2, (0, 0, 0))]


def g2slot(f: int) -> int:
    return 0 if f == 0 else (1 if f == 1 else (2 + f - 3 if f < 9 else 8 + f - 9))


def _exponent(m: np.ndarray) -> np.ndarray:
    e = np.zeros(m.shape, dtype=np.int64)
    nz = m > 0
    e[nz] = np.frexp(m[nz])[1].astype(np.int64) + 1
    return e


def _band(digits: np.ndarray, coef: np.ndarray, R: int) -> np.ndarray:
    """Exact integer stencil sums: out[..., o] = sum_j coef[j] digits[..., o + R + j - len(coef)//2]."""
    half = len(coef) // 2
    out = np.zeros(digits.shape[:-1] + (NO,), dtype=np.int64)
    for j, c in enumerate(coef):
        if c:
            start = R - half + j
            out += c * digits[..., start:start + NO]
    return out


def _recombine(acc: np.ndarray, k: int) -> np.ndarray:
    """Planes in pairs from the smallest, r = r + (acc_{s-1} 128 + acc_s) 2^(-7(s+1))
    in float64 (the pair is an exact integer), an odd top plane alone."""
    r = np.zeros(acc.shape[1:], dtype=np.float64)
    w = math.ldexp(1.0, -7 * k)
    s = k - 1
    while s >= 1:
        r = r + (acc[s - 1] * 128 + acc[s]).astype(np.float64) * w
        w *= 16384.0
        s -= 2
    if s == 0:
        r = r + acc[0].astype(np.float64) * w
    return r


def ozaki_pass(F: np.ndarray, axis: int, k: int, h: float, want_d2: bool, ko_R: int = 0,
               ko_sigma: float = 0.0, core: int = 0, ext=(0, 0, 0)):
    """One pass over the 3D array F: (d1, d2, ko) on the covered box (NaN
    elsewhere; d2 / ko are None when not formed). ko_R = 3 (KO6), 4 (KO8)
    or 0 (no KO term)."""
    R = 4 if ko_R == 4 else 3
    KWL = NO + 2 * R
    s = F.shape
    m = [max(core - x, 0) for x in ext]
    box = tuple(slice(m[q], s[q] - m[q]) for q in range(3))
    # the box's lines along the axis: (..., len) with the axis last
    A = np.moveaxis(F, axis, -1)
    other = [q for q in range(3) if q != axis]
    A = A[box[other[0]], box[other[1]], :]
    lines = A.reshape(-1, s[axis])
    L = s[axis] - 2 * m[axis]
    nzt = -(-L // NO)
    z0 = np.arange(nzt) * NO
    pos = m[axis] + z0[:, None] - R + np.arange(KWL)[None, :]
    win = lines[:, np.clip(pos, 0, s[axis] - 1)]  # (nlines, nzt, KWL)
    e = _exponent(np.abs(win).max(axis=2))
    y = win * np.ldexp(1.0, -e)[..., None]
    X = np.rint(y * math.ldexp(1.0, 7 * k)).astype(np.int64)
    digits = np.stack([X >> (7 * (k - 1)) if s2 == 0 else (X >> (7 * (k - 1 - s2))) & 127
                       for s2 in range(k)])  # (k, nlines, nzt, KWL)
    sc = np.ldexp(1.0, e)[..., None]
    out = {}
    r1 = _recombine(_band(digits, C1, R), k)
    out["d1"] = (r1 * sc) * ((1.0 / 60.0) * (1.0 / h))
    if want_d2:
        acc2 = _band(digits, C2H, R) * 128 + _band(digits, C2L, R)
        out["d2"] = (_recombine(acc2, k) * sc) * ((1.0 / 180.0) * (1.0 / (h * h)))
    if ko_R:
        kc = K8 if ko_R == 4 else K6
        den = 256.0 if ko_R == 4 else 64.0
        out["ko"] = (_recombine(_band(digits, kc, R), k) * sc) * ((1.0 / den) * (ko_sigma / h))
    res = []
    for name in ("d1", "d2", "ko"):
        if name not in out:
            res.append(None)
            continue
        v = out[name].reshape(lines.shape[0], nzt * NO)[:, :L]
        full = np.full(F.shape, np.nan)
        view = np.moveaxis(full, axis, -1)
        sub = v.reshape(A.shape[0], A.shape[1], L)
        view[box[other[0]], box[other[1]], m[axis]:s[axis] - m[axis]] = sub
        res.append(full)
    return tuple(res)


def bundle(F: np.ndarray, h, k: int, ko_sigma: float = 0.0, ko_order: int = 6, core: int = 0) -> np.ndarray:
    """The 138 derivatives (+24 KO sums with ko_sigma > 0) of F (24, sx, sy, sz)
    through the Ozaki passes; NaN where a slot is not formed."""
    hs = (h, h, h) if np.isscalar(h) else tuple(h)
    use_ko = ko_sigma > 0
    nslot = 162 if use_ko else 138
    D = np.full((nslot,) + F.shape[1:], np.nan)
    diag = [0, 3, 5]
    for f in range(24):
        d2f = f in D2_FIELDS
        for axis in range(3):
            kind = (0 if d2f else 1) if axis == 0 else ((2 if d2f else 3) if axis == 1 else 4)
            ko_R = (4 if ko_order == 8 else 3) if use_ko else 0
            d1, d2, ko = ozaki_pass(F[f], axis, k, hs[axis], d2f, ko_R, ko_sigma, core, KINDS[kind][1])
            D[3 * f + axis] = d1
            if d2f:
                D[72 + 6 * g2slot(f) + diag[axis]] = d2
            if use_ko:
                D[138 + f] = ko if axis == 0 else D[138 + f] + ko
    for f in D2_FIELDS:
        g = 72 + 6 * g2slot(f)
        D[g + 1] = ozaki_pass(D[3 * f + 0], 1, k, hs[1], False, 0, 0.0, core, KINDS[3][1])[0]
        D[g + 2] = ozaki_pass(D[3 * f + 0], 2, k, hs[2], False, 0, 0.0, core, KINDS[4][1])[0]
        D[g + 4] = ozaki_pass(D[3 * f + 1], 2, k, hs[2], False, 0, 0.0, core, KINDS[4][1])[0]
    return D
