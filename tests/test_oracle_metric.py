"""The grouped error metric of the oracle (per field, scaled by its tensor)."""

import numpy as np

from oracle import oracle as O


def test_grouped_metric_uses_tensor_scale():
    b = np.zeros((24, 4))
    b[3] = 1.0            # gt0 ~ 1
    b[4] = 1e-8           # gt1: noise-level off-diagonal entry
    a = b.copy()
    a[4] += 1e-20
    assert O.normwise_rel(a, b)[4] > 1e-13            # per field: 1e-12 relative to 1e-8
    assert O.normwise_rel_grouped(a, b)[4] < 1e-19    # grouped: relative to the tensor (gt0 ~ 1)
    a[0] += 1.0
    assert O.normwise_rel_grouped(a, b)[0] == 1.0 / 1e-300 or O.normwise_rel_grouped(a, b)[0] > 1e100
