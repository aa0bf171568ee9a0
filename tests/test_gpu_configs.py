"""GPU parity at the sizes of the benchmark configurations.

Config 3 (the batched workload, mix20k: 20,909 blocks, 87.0 M zones): ten
graph-replayed RK4 steps through the plan with the right-hand side tiles the
autotuner picks, constraint L2 norms by the plan's in-graph diagnostics
after every second step, against the norms the reference's own compiled
right-hand side produced on the CPU (tests/golden/config3_norms.json,
make_config3_golden.py), to 1e-10.

Config 2 (the mixed-size octree at the plain-path size): 4,108 blocks of
sides 13..55 with the configured size mix, ten graph-replayed RK4 steps
(ghost fill, right-hand side, zip, stage algebra, enforcement) from the
oracle's initial state, against the state and the constraint-norm history
that the reference's own compiled right-hand side produced on the CPU
(tests/golden/config2_golden.npz, make_config2_golden.py): every variable at
4,096 seeded nodes relative to the variable's largest magnitude, the largest
magnitudes and sums of squares over all nodes, and the Hamiltonian and
momentum constraint L2 norms after every step.  Run once with the split
right-hand side and once with the on-chip one."""
import os

import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "config2_golden.npz")

# per-variable error after ten steps relative to the variable's largest
# magnitude; the constraint norms relative to themselves
TOL_STATE = 1e-12
TOL_NORMS = 1e-10


def _onchip_tiles(B):
    pick = {}
    for t, shape in enumerate(B.tiles()):
        if B.tile_mode(t) == 2:
            pick.setdefault(shape[:3], []).append(t)
    return {13: pick[(7, 4, 4)][0], 19: pick[(5, 5, 5)][0], 31: pick[(5, 5, 5)][0], 55: pick[(5, 5, 5)][0]}


@pytest.mark.parametrize("rhs", ["split", "onchip"])
def test_config2_ten_steps_vs_reference(rhs):
    import bssn_b200 as B
    gold = np.load(GOLD)
    spec = B.generate_mesh(1, tuple(int(x) for x in gold["dims"]), seed=int(gold["seed"]),
                           L=float(gold["L"]), origin=tuple(float(x) for x in gold["origin"]))
    assert spec.nblocks == int(gold["nblocks"]) and spec.zones() == int(gold["zones"])
    mo = ol.MeshOracle(spec, ol.oracle())
    bh = tuple(float(x) for x in gold["bh"])
    U = torch.from_numpy(mo.initial_data(bh=bh, eps=1e-8)).cuda()
    m = B.Mesh(spec)
    plan = B.RK4Plan(m, B.default_params(), B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH)
    if rhs == "onchip":
        for side, t in _onchip_tiles(B).items():
            plan.set_tile(t, side)
    Pz = torch.zeros((24, m.n_unzip), dtype=torch.float64, device="cuda")
    cons = torch.zeros((4, spec.n_nodes), dtype=torch.float64, device="cuda")
    norms = torch.zeros(4, dtype=torch.float64, device="cuda")

    def measure():
        m.unzip(Pz, U)
        B.constraints(m, cons, Pz)
        B.constraint_norms(m, cons, norms, bh=bh, radii=(0.5, 0.5))
        torch.cuda.synchronize()
        return norms.cpu().numpy().copy()

    hist = [measure()]
    dt = 0.25 * spec.h
    for _ in range(int(gold["steps"])):
        plan.step(U, dt)
        hist.append(measure())
    assert plan.violations() == int(gold["enforce_violations"])
    plan.close()
    idx = torch.from_numpy(gold["sample_idx"]).cuda()
    got = U[:, idx].cpu().numpy()
    scale = gold["maxabs"]
    err = (np.abs(got - gold["sample"]).max(axis=1) / scale)
    assert err.max() <= TOL_STATE, {v: float(e) for v, e in enumerate(err) if e > TOL_STATE}
    maxabs = U.abs().max(dim=1).values.cpu().numpy()
    sumsq = (U * U).sum(dim=1).cpu().numpy()
    assert (np.abs(maxabs - scale) / scale).max() <= TOL_STATE
    assert (np.abs(sumsq - gold["sumsq"]) / gold["sumsq"]).max() <= 2 * TOL_STATE
    rel = np.abs(np.array(hist) - gold["norms"]) / np.abs(gold["norms"])
    assert rel.max() <= TOL_NORMS, rel.max(axis=1)


def test_config3_norms_mix20k():
    import json
    import bssn_b200 as B
    path = os.path.join(HERE, "golden", "config3_norms.json")
    with open(path) as f:
        gold = json.load(f)
    spec = B.generate_mesh(1, (10, 10, 7), seed=20261203)
    assert spec.nblocks == gold["nblocks"] and spec.zones() == gold["zones"]
    mo = ol.MeshOracle(spec, ol.oracle())
    U = torch.from_numpy(mo.initial_data(eps=1e-8)).cuda()
    m = B.Mesh(spec)
    plan = B.RK4Plan(m, B.default_params(), B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH)
    plan.autotune(U, reps=1)
    norms = torch.zeros(4, dtype=torch.float64, device="cuda")
    dt = 0.25 * spec.h
    got = {}
    plan.diagnostics(U, norms)
    torch.cuda.synchronize()
    got[0] = norms.cpu().numpy().copy()
    for step in range(1, 11):
        plan.step(U, dt)
        if step % 2 == 0:
            plan.diagnostics(U, norms)
            torch.cuda.synchronize()
            got[step] = norms.cpu().numpy().copy()
    assert plan.violations() == gold["enforce_violations"]
    plan.close()
    worst = 0.0
    for h in gold["history"]:
        ref = np.array([float.fromhex(x) for x in h["norms"]])
        worst = max(worst, (np.abs(got[h["step"]] - ref) / np.abs(ref)).max())
    assert worst <= TOL_NORMS, worst
