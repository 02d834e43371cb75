"""A minimal stand-in for the ``jax`` package, used only to run the
reference's M4 kernel generator (3D/src/bssn3d/cuda/gen_fused.py) unchanged
where JAX is not installed. The generator needs three things from JAX at
import time: ``jax.config.update("jax_enable_x64", True)`` (gen_fused.py:26-27),
and ``jax.numpy.array`` / ``jax.lax`` for the stencil tables of
``mcs_common.derivatives.SpatialDerivative`` (derivatives.py:13-14,35-49),
which the generator reads with ``np.asarray`` (gen_fused.py:183-185). numpy
float64 arrays give the same coefficient values as JAX in x64 mode.
Nothing else of JAX is provided; this package is never on the product path.
"""

from . import lax, numpy  # noqa: F401


class _Config:
    def update(self, name, value):
        # x64 is numpy's default; nothing to switch
        return None


config = _Config()
