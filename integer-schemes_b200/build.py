"""Build the sm_100a CUDA library in-tree.

    python integer-schemes_b200/build.py          # libbssn_b200.so (+ -Xptxas -v report)

Extra nvcc flags (e.g. -DBSSN_B200_NO_TMA) can be given in $BSSN_B200_NVCC_FLAGS.

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

SOURCES = [CSRC / "bssn_b200.cu", CSRC / "stream_rhs.cu", CSRC / "stream_stage.cu", CSRC / "stream_msrk.cu",
           CSRC / "stream_batch3.cu", CSRC / "stream_batch4.cu", CSRC / "ozaki.cu", CSRC / "amr_fill.cu"]
OBJ_DIR = HERE / "_build"
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


def _compile(src: Path) -> tuple:
    obj = OBJ_DIR / (src.stem + ".o")
    cmd = [nvcc(), *ARCH, *host_compiler(), "-O3", "-lineinfo", "-std=c++17",
           "-Xptxas", "-v", "-Xcompiler", "-fPIC", "-diag-suppress", "177",
           *os.environ.get("BSSN_B200_NVCC_FLAGS", "").split(),
           "-c", str(src), "-o", str(obj)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    return src, obj, proc


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile every translation unit in parallel, then link the shared library."""
    if not force and up_to_date():
        return LIB
    from concurrent.futures import ThreadPoolExecutor
    OBJ_DIR.mkdir(exist_ok=True)
    workers = max(1, min(len(SOURCES), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as pool:
        results = list(pool.map(_compile, SOURCES))
    report = []
    for src, obj, proc in results:
        report.append(proc.stderr)
        if proc.returncode != 0:
            sys.stderr.write(proc.stdout + proc.stderr)
            raise RuntimeError(f"nvcc failed on {src.name} ({proc.returncode})")
    link = [nvcc(), *ARCH, *host_compiler(), "-shared", "-o", str(LIB), *[str(o) for _, o, _ in results]]
    proc = subprocess.run(link, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError(f"link failed ({proc.returncode})")
    text = "".join(report)
    (PKG / "ptxas_report.txt").write_text(text)
    if verbose:
        sys.stdout.write(text)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
