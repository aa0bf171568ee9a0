"""Restart from a checkpoint on the GPU: an evolution written to disk after
k steps, restored into a fresh mesh and plan and continued, ends bit-identical
to the same evolution run without interruption (the reference's
restore_checkpt contract, BSSN_GR/src/bssnCtx.cpp:864-1170: the restored
state and time-stepper resume where the checkpoint was taken)."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def B():
    import bssn_b200
    return bssn_b200


def evolve(B, spec, U, steps, dt):
    m = B.Mesh(spec)
    plan = B.RK4Plan(m, B.default_params(), B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH)
    for _ in range(steps):
        plan.step(U, dt)
    torch.cuda.synchronize()
    plan.close()
    m.close()


def test_restart_is_bit_identical(B, tmp_path):
    from bssn_b200 import checkpoint as ck
    spec = B.generate_mesh(1, (1, 1, 1), seed=8, xmin=-8.25)
    dt = 0.25 * spec.h
    U = torch.zeros((24, spec.n_nodes), dtype=torch.float64, device="cuda")
    B.initial_data(U, spec)
    evolve(B, spec, U, 2, dt)
    prefix = str(tmp_path / "bssn")
    idx = ck.write_checkpoint(prefix, spec, U, step=2, time=2 * dt, dt=dt, freq=1)
    U_cp = U.clone()
    evolve(B, spec, U, 2, dt)          # uninterrupted: steps 3 and 4
    spec2, V, info = ck.restore_checkpoint(prefix)
    assert info.step == 2 and info.time_step == dt and idx == 0
    assert torch.equal(V, U_cp)
    evolve(B, spec2, V, 2, info.time_step)   # restarted: steps 3 and 4
    assert torch.equal(V.view(torch.int64), U.view(torch.int64))
    assert np.isfinite(U.cpu().numpy()).all()
