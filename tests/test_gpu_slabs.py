"""Slab split of one uniform block on the GPU, every rank's slab stepped by
one process on one device (the distributed run's schedule: per stage, each
slab's fused stage launch, then the halo planes copied from the
neighbours' owned planes). The owned planes equal the single-block
evolution bit for bit, and the slab constraint norms (per-slab constraint
launch, sums over the owned interior planes) agree with the single-block
norm kernel to rounding."""

import pytest
import torch

pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.mark.parametrize("n,world,ko_order,ng", [(24, 2, 6, 3), (24, 3, 6, 3), (40, 4, 8, 4), (128, 2, 6, 3)])
def test_slabs_step_like_one_block(n, world, ko_order, ng):
    from bssn3d_b200 import initial_data as ID
    from bssn3d_b200.constraints import ConstraintSolver
    from bssn3d_b200.evolve import BSSNEvolution
    from bssn3d_b200.slabs import SlabEvolution
    grid, U_host, dt = ID.workload(1, n=n, ng=ng)
    U = torch.from_numpy(U_host).to(DEV)
    evo = BSSNEvolution(grid, ko_sigma=0.1, bc="none", ko_order=ko_order)
    nsteps = 2
    want = U.clone()
    S = evo._S(0.0, dt, U.device)
    for _ in range(nsteps):
        evo._step_inplace(want, S)
        evo._advance_time(S)
    slabs = [SlabEvolution(grid, world=world, rank=r, ko_sigma=0.1, ko_order=ko_order) for r in range(world)]
    got = SlabEvolution.evolve_in_one_process(slabs, [s.local(U) for s in slabs], dt, nsteps)
    torch.cuda.synchronize()
    for s, G in zip(slabs, got):
        lay = s.layout
        assert torch.equal(s.owned(G), want[:, lay.a:lay.b]), f"rank {lay.rank} owned planes differ"
        assert torch.equal(G, want[:, lay.local_slice()]), f"rank {lay.rank} halo planes stale"
    # norms: every slab's sums over its owned interior planes, added as the all-reduce would
    h_ref, m_ref = ConstraintSolver(grid).l2(want)
    sums = sum(s.constraint_sums(G).cpu() for s, G in zip(slabs, got))
    h, m = torch.sqrt(sums[:2] / sums[2]).tolist()
    assert abs(h - h_ref) <= 1e-12 * h_ref and abs(m - m_ref) <= 1e-12 * m_ref
