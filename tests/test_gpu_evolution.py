"""GPU: 100 RK4 steps of the uniform 512-block 13^3 workload through the
batched, graph-captured plan; the Hamiltonian and momentum constraint L2
norms every 10 steps must match, to 1e-10 relative, the history the
reference's own right-hand side produced on the CPU
(tests/golden/constraint_history.json, make_constraint_golden.py)."""
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
HERE = os.path.dirname(os.path.abspath(__file__))


def test_constraint_norm_history_100_steps():
    import bssn_b200 as B
    with open(os.path.join(HERE, "golden", "constraint_history.json")) as f:
        gold = json.load(f)
    spec = B.generate_mesh(0, (8, 8, 8))
    m = B.Mesh(spec)
    U = torch.zeros((24, spec.n_nodes), dtype=torch.float64, device="cuda")
    B.initial_data(U, spec)
    dt = 0.25 * spec.h
    plan = B.RK4Plan(m, B.default_params(), B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH)
    Pz = torch.zeros((24, m.n_unzip), dtype=torch.float64, device="cuda")
    cons = torch.zeros((4, spec.n_nodes), dtype=torch.float64, device="cuda")
    norms = torch.zeros(4, dtype=torch.float64, device="cuda")

    def measure():
        m.unzip(Pz, U)
        B.constraints(m, cons, Pz)
        B.constraint_norms(m, cons, norms, radii=(0.5, 0.5))
        torch.cuda.synchronize()
        return norms.cpu().numpy().copy()

    got = {0: measure()}
    for step in range(1, 101):
        plan.step(U, dt)
        if step % 10 == 0:
            got[step] = measure()
    assert plan.violations() == gold["enforce_violations"]
    worst = 0.0
    for h in gold["history"]:
        ref = np.array([float.fromhex(x) for x in h["norms"]])
        rel = np.abs(got[h["step"]] - ref) / np.abs(ref)
        worst = max(worst, rel.max())
    assert worst <= 1e-10, worst


def test_constraint_norm_history_in_graph():
    """The same history through the plan's graph-captured step + diagnostics
    (bssn_rk4_plan_step_diag every 10th step, norms copied on the device into
    a history tensor): one host synchronisation at the end, same norms."""
    import bssn_b200 as B
    with open(os.path.join(HERE, "golden", "constraint_history.json")) as f:
        gold = json.load(f)
    spec = B.generate_mesh(0, (8, 8, 8))
    m = B.Mesh(spec)
    U = torch.zeros((24, spec.n_nodes), dtype=torch.float64, device="cuda")
    B.initial_data(U, spec)
    dt = 0.25 * spec.h
    plan = B.RK4Plan(m, B.default_params(), B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH)
    norms = torch.zeros(4, dtype=torch.float64, device="cuda")
    hist = torch.zeros((11, 4), dtype=torch.float64, device="cuda")
    plan.diagnostics(U, norms)
    hist[0].copy_(norms)
    for step in range(1, 101):
        if step % 10 == 0:
            plan.step_diag(U, dt, norms)
            hist[step // 10].copy_(norms)
        else:
            plan.step(U, dt)
    got = hist.cpu().numpy()
    assert plan.violations() == gold["enforce_violations"]
    worst = 0.0
    for h in gold["history"]:
        ref = np.array([float.fromhex(x) for x in h["norms"]])
        worst = max(worst, (np.abs(got[h["step"] // 10] - ref) / np.abs(ref)).max())
    assert worst <= 1e-10, worst


def test_psi4_in_diagnostics_graph():
    """With PLAN_DIAG_PSI4 the graph-captured step + diagnostics also
    writes psi4: the plan's fields equal bssn_constraints_psi4_f64 on the
    ghost-filled new state (same kernel, bit for bit), and feed the
    gravitational-wave extraction directly."""
    import ctypes as C
    import bssn_b200 as B
    from bssn_b200 import gw
    spec = B.generate_mesh(1, (2, 1, 1), seed=1, xmin=-8.25)
    m = B.Mesh(spec)
    U = torch.zeros((24, spec.n_nodes), dtype=torch.float64, device="cuda")
    B.initial_data(U, spec)
    plan = B.RK4Plan(m, B.default_params(), B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH | B.PLAN_DIAG_PSI4)
    norms = torch.zeros(4, dtype=torch.float64, device="cuda")
    for _ in range(2):
        plan.step_diag(U, 0.25 * spec.h, norms)
    fields = plan.diag_fields(torch.empty((6, spec.n_nodes), dtype=torch.float64, device="cuda"))
    P = torch.zeros((24, m.n_unzip), dtype=torch.float64, device="cuda")
    m.unzip(P, U)
    ref = torch.zeros((6, spec.n_nodes), dtype=torch.float64, device="cuda")
    cp = (C.c_void_p * 6)(*[ref[c].data_ptr() for c in range(6)])
    B.lib.bssn_constraints_psi4_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
    assert B.lib.bssn_constraints_psi4_f64(m.h, B.ptrs(P), cp, B.stream_ptr()) == 0
    torch.cuda.synchronize()
    assert torch.equal(fields, ref)
    md, coeff, l2 = gw.extract(fields[4].contiguous(), fields[5].contiguous(), spec, (3.0, 5.0), lmax=3)
    assert np.isfinite(coeff).all() and (l2 > 0).all()
