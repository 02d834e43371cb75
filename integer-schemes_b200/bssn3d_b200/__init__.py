"""bssn3d_b200 — the bssn3d BSSN right-hand side and RK4 stage update on
NVIDIA B200 (sm_100a).

Host-side mirror of the reference's bssn3d interface for this path:

* ``fused_rhs.cuda_fused_algebra`` — the fused-RHS callable
  (3D/src/bssn3d/fused_rhs_cuda.py:62-72)
* ``rhs.BSSNSolver`` — the RHS entry point (3D/src/bssn3d/rhs.py:63-139)
* ``evolve.BSSNEvolution`` — RK4 + KO + enforcement (3D/src/bssn3d/evolve.py:24-194)
* ``state``, ``grid``, ``initial_data`` — state container, grid, input data

Compute runs only in ``libbssn_b200.so`` (C ABI: include/bssn_b200.h).
"""

from .state import (BSSNState, PhysicsParams, VAR_NAMES, FIELD_INPUTS, OUTPUT_FIELDS,
                    NUM_VARS)
from .grid import Grid

__all__ = ["BSSNState", "PhysicsParams", "VAR_NAMES", "FIELD_INPUTS", "OUTPUT_FIELDS",
           "NUM_VARS", "Grid"]
