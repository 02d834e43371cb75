"""HostStepPipeline: a stream of host-resident states, each advanced by one
RK4 step with the copies overlapped with the compute, gives exactly the
states BSSNEvolution.step gives one at a time."""

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nslots", [1, 2, 3])
def test_pipelined_host_steps_equal_single_steps(nslots):
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.evolve import BSSNEvolution, HostStepPipeline
    from bssn3d_b200.state import BSSNState
    grid, U, dt = ID.workload(1, n=20)
    evo = BSSNEvolution(grid, ko_sigma=0.1, bc="none", ko_order=6)
    rng = np.random.default_rng(4)
    states = [U + 1e-4 * rng.standard_normal(U.shape) * (k > 0) for k in range(5)]
    host_in = [torch.from_numpy(s).pin_memory() for s in states]
    host_out = [torch.empty_like(h).pin_memory() for h in host_in]
    pipe = HostStepPipeline(evo, U.shape, dt, 0.3, nslots=nslots)
    pipe.run(host_in, host_out)
    torch.cuda.synchronize()
    for s, h in zip(states, host_out):
        ref = evo.step(BSSNState(torch.from_numpy(s).cuda()), 0.3, dt).data.cpu()
        assert torch.equal(h, ref)
