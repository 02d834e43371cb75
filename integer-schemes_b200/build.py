"""Build the sm_100a CUDA library in-tree.

    python integer-schemes_b200/build.py          # libbssn_b200.so (+ -Xptxas -v report)

The library lands next to the Python package that loads it
(``bssn3d_b200/libbssn_b200.so``), so it travels with the source tree.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
PKG = HERE / "bssn3d_b200"
LIB = PKG / "libbssn_b200.so"
ROOT = HERE.parent

SOURCES = [CSRC / "bssn_b200.cu", CSRC / "ozaki.cu", CSRC / "amr_fill.cu"]
HEADERS = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "bssn_b200.h"]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise FileNotFoundError("nvcc not found")


def host_compiler() -> list:
    # the system g++ (an environment CXX may point at a toolchain without libgomp)
    for cand in ("/usr/bin/g++",):
        if Path(cand).exists():
            return ["-ccbin", cand]
    return []


def up_to_date() -> bool:
    if not LIB.exists():
        return False
    t = LIB.stat().st_mtime
    return all(p.stat().st_mtime <= t for p in SOURCES + HEADERS + [Path(__file__)])


def build(verbose: bool = False, force: bool = False) -> Path:
    if not force and up_to_date():
        return LIB
    cmd = [nvcc(), *ARCH, *host_compiler(), "-O3", "-lineinfo", "-std=c++17",
           "-Xptxas", "-v", "-shared", "-Xcompiler", "-fPIC",
           "-diag-suppress", "177",
           "-o", str(LIB), *map(str, SOURCES)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError(f"nvcc failed ({proc.returncode})")
    report = PKG / "ptxas_report.txt"
    report.write_text(proc.stderr)
    if verbose:
        sys.stdout.write(proc.stderr)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
