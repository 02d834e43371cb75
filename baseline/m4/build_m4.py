"""Build the reference's M4 fused BSSN RHS kernel for sm_100a (baseline only).

    python baseline/m4/build_m4.py [--reference ROOT]

The reference root comes from ``--reference`` or the environment variable
``INTEGER_SCHEMES_REFERENCE``; with neither, the read-only mount the reference
is provided at in this build container is used. Steps:

1. run the reference's generator 3D/src/bssn3d/cuda/gen_fused.py unchanged
   (its default settings: per-tap loads, no shared-memory parking) with the
   jax stand-in of baseline/m4/jax_stand_in on the path (JAX is not installed
   here), writing the generated kernel to baseline/_ref/m4/_bssn_fused_kernel.cuh;
2. compile baseline/m4/m4_launch.cu against it for sm_100a into
   baseline/_ref/m4/libm4_rhs.so (plus the -Xptxas -v report beside it).

baseline/_ref/ is git-ignored: the generated source is the reference's, not
this project's, and only the built library travels to the GPU machine.
"""

from __future__ import annotations

import argparse
import importlib.util
import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
OUT = ROOT / "baseline" / "_ref" / "m4"
DEFAULT_REFERENCE = "/root/reference"


def generate(reference: Path, header: Path) -> None:
    src3d = reference / "3D" / "src"
    common = reference / "common" / "src"
    for p in (str(HERE / "jax_stand_in"), str(src3d), str(common)):
        if p not in sys.path:
            sys.path.insert(0, p)
    spec = importlib.util.spec_from_file_location(
        "bssn3d.cuda.gen_fused", src3d / "bssn3d" / "cuda" / "gen_fused.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    for knob in ("BSSN_FUSED_V7", "BSSN_FUSED_SMEM_K"):
        os.environ.pop(knob, None)   # the generator's defaults
    mod.generate(header)


def main() -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference", default=os.environ.get("INTEGER_SCHEMES_REFERENCE", DEFAULT_REFERENCE))
    args = ap.parse_args()
    reference = Path(args.reference)
    if not (reference / "3D" / "src" / "bssn3d" / "cuda" / "gen_fused.py").exists():
        print(f"reference tree not found at {reference}", file=sys.stderr)
        return 2
    OUT.mkdir(parents=True, exist_ok=True)
    header = OUT / "_bssn_fused_kernel.cuh"
    generate(reference, header)
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    lib = OUT / "libm4_rhs.so"
    cmd = [nvcc, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-lineinfo", "-std=c++17",
           "-Xptxas", "-v", "-shared", "-Xcompiler", "-fPIC", "-I", str(OUT),
           "-o", str(lib), str(HERE / "m4_launch.cu")]
    if Path("/usr/bin/g++").exists():
        cmd[1:1] = ["-ccbin", "/usr/bin/g++"]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    (OUT / "ptxas_report.txt").write_text(proc.stderr)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        return proc.returncode
    print(lib)
    return 0


if __name__ == "__main__":
    sys.exit(main())
