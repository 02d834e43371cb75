"""Algorithmic FP64 flop count of one BSSN right-hand-side point-update.

Build-time tool (it reads the reference tree, which only this container
has): counts the arithmetic of the reference's vendored Dendro-GR CSE
(3D/src/bssn3d/vendor/bssneqs_SSL_HD_dxsq.cpp, the algebra the fused kernel
restates) statement by statement — binary +, -, *, / (a fraction of two
numeric literals is folded at compile time and not counted), integer pow()
lowered to repeated multiplication (a negative power adds one division),
sqrt and exp one each — and adds the separable derivative count and the KO6
taps. bench.py pins the result as FLOPS_PER_POINT and KO_FLOPS_PER_POINT.

    python oracle/count_flops.py [path/to/bssneqs_SSL_HD_dxsq.cpp]

Without an argument the file is taken from the reference root named by
$INTEGER_SCHEMES_REFERENCE, else from the read-only mount the reference has
in the build container.
"""

from __future__ import annotations

import os
import re
import sys
from pathlib import Path

DEFAULT = Path(os.environ.get("INTEGER_SCHEMES_REFERENCE", "/root/reference")) / "3D/src/bssn3d/vendor/bssneqs_SSL_HD_dxsq.cpp"

_LIT = r"\d+(?:\.\d*)?(?:[eE][-+]?\d+)?"
_FRACTION = re.compile(rf"\(\s*{_LIT}\s*/\s*{_LIT}\s*\)")
_POW = re.compile(r"pow\(\s*([^,()]+(?:\[[^\]]*\])?)\s*,\s*(-?\d+)\s*\)")


def _rhs_statements(text: str):
    for line in text.splitlines():
        line = line.strip()
        if line.startswith("//") or "=" not in line or not line.endswith(";"):
            continue
        lhs, rhs = line[:-1].split("=", 1)
        if "==" in line or not lhs.strip():
            continue
        yield rhs


def count_algebra(text: str) -> dict:
    c = {"add": 0, "sub": 0, "neg": 0, "mul": 0, "div": 0, "pow": 0, "sqrt": 0, "exp": 0}
    for rhs in _rhs_statements(text):
        for m in _POW.finditer(rhs):
            n = int(m.group(2))
            c["pow"] += abs(n) - 1 + (1 if n < 0 else 0)
        rhs = _POW.sub("P", rhs)
        rhs = _FRACTION.sub("L", rhs)
        c["sqrt"] += len(re.findall(r"\bsqrt\(", rhs))
        c["exp"] += len(re.findall(r"\bexp\(", rhs))
        toks = re.findall(rf"[A-Za-z_]\w*(?:\[[^\]]*\])?|{_LIT}|[-+*/()]", rhs)
        prev = None  # an operand or ')' before a sign makes it binary
        for i, t in enumerate(toks):
            if t in "+-":
                if prev is not None and prev not in "+-*/(":
                    c["add" if t == "+" else "sub"] += 1
                elif t == "-" and i + 1 < len(toks) and not re.fullmatch(_LIT, toks[i + 1]):
                    c["neg"] += 1  # a sign in front of a literal is part of the constant
            elif t == "*":
                c["mul"] += 1
            elif t == "/":
                c["div"] += 1
            prev = t
    # negations are reported but not counted: they fold into the sign of a
    # neighbouring multiply, add or fused multiply-add
    c["algebra"] = c["add"] + c["sub"] + c["mul"] + c["div"] + c["pow"] + c["sqrt"] + c["exp"]
    return c


def count_derivatives() -> int:
    """Separable minimum: 72 first derivatives (6 nonzero taps: 6 mul + 5 add,
    + 1 scale + 1 for the pre-scaled weight = 13), 18 diagonal second (7 taps:
    7 mul + 6 add + 1 scale = 14), 48 mixed as two first-derivative passes
    (26)."""
    return 72 * 13 + 18 * 14 + 48 * 26


def count_ko6() -> int:
    """24 fields x 3 axes x (7 taps: 7 mul + 6 add)."""
    return 24 * 3 * 13


def main(argv) -> int:
    path = Path(argv[1]) if len(argv) > 1 else DEFAULT
    c = count_algebra(path.read_text())
    d = count_derivatives()
    print(f"algebra: {c['add']} add + {c['sub']} sub + {c['mul']} mul + {c['div']} div + {c['pow']} from pow "
          f"+ {c['sqrt']} sqrt + {c['exp']} exp = {c['algebra']} ({c['neg']} negations not counted)")
    print(f"derivatives (separable): {d}")
    print(f"RHS per point-update: {c['algebra'] + d}; KO6: {count_ko6()}")
    return 0


if __name__ == "__main__":
    sys.exit(main(sys.argv))
