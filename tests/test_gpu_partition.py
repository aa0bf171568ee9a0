"""The partitioned GPU evolution (bssn_b200.distributed.PartitionedRK4):
two ranks as two processes sharing one GPU, their halo exchange over gloo
through host memory (no kernel of one process waits on the other).  The
owned nodes after two RK4 steps must equal the single-domain plan's result
bit for bit (same kernels, same data)."""
import tempfile

import numpy as np
import pytest

import oracle_lib as ol
import partition_ranks as pr
from test_partition import gather, run_ranks

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.mark.parametrize("kind", ["uniform", "mix"])
def test_partitioned_gpu_step_matches_single_domain(kind):
    import bssn_b200 as B
    world, steps = 2, 2
    spec = pr.mesh(kind)
    Z0 = ol.MeshOracle(spec, ol.oracle()).initial_data(eps=1e-8)
    m = B.Mesh(spec)
    plan = B.RK4Plan(m, B.default_params(), B.PLAN_ENFORCE_STAGES)
    U = torch.from_numpy(Z0).cuda()
    for _ in range(steps):
        plan.step(U, 0.25 * spec.h)
    norms = torch.zeros(4, dtype=torch.float64, device="cuda")
    plan.diagnostics(U, norms)
    torch.cuda.synchronize()
    ref = U.cpu().numpy()
    ref_norms = norms.cpu().numpy()
    plan.close()
    m.close()
    with tempfile.TemporaryDirectory() as d:
        run_ranks(pr.gpu_rank, world, kind, steps, d)
        ids, vals = gather(d, world)
        got_norms = [np.load(f"{d}/norms{r}.npy") for r in range(world)]
    assert len(np.unique(np.concatenate(ids))) == spec.n_nodes
    for i, v in zip(ids, vals):
        assert np.array_equal(v, ref[:, i])
    # norms from owned-node sums reduced over the ranks (different summation
    # order than the single domain's reduction)
    for n in got_norms:
        assert np.allclose(n, ref_norms, rtol=1e-12, atol=0), (n, ref_norms)
