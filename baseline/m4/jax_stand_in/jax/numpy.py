"""numpy in place of jax.numpy for the generator's stencil tables."""

from numpy import *  # noqa: F401,F403
from numpy import array, ndarray  # noqa: F401
