"""Multi-level meshes on the GPU against the level oracle (oracle_levels.py):
ghost fill with coarse-to-fine interpolation and the level sync bit-exact,
initial data per level grid, and RK4 steps of the plan (ghost fill,
right-hand side per block at its level's spacing, owner gather, node-wise
stage, level sync) within the tolerances of the single-level tests."""
import numpy as np
import pytest

import oracle_lib as ol
from oracle_levels import LevelOracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

MESHES = {
    "two": ((4, 4, 4), [((2, 2, 2), (4, 4, 4))]),
    "three": ((6, 6, 6), [((2, 4, 2), (6, 4, 8)), ((6, 10, 6), (4, 2, 6))]),
}


@pytest.fixture(scope="module")
def O():
    return ol.oracle()


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def setup(name, O):
    import bssn_b200 as B
    from bssn_b200 import levels as LV
    M0, boxes = MESHES[name]
    spec = LV.generate_levels(M0, boxes)
    return B, LV, spec, LevelOracle(spec, O)


@pytest.mark.parametrize("name", sorted(MESHES))
def test_ghost_fill_and_sync_bit_exact(name, O):
    B, LV, spec, LO = setup(name, O)
    rng = np.random.default_rng(3)
    Z = rng.standard_normal((24, spec.n_nodes))
    m = B.Mesh(spec)
    P = torch.zeros((24, m.n_unzip), dtype=torch.float64, device="cuda")
    dZ = dev(Z)
    m.unzip(P, dZ)
    LV.sync(m, dZ)
    torch.cuda.synchronize()
    ref_p = LO.unzip(Z)
    ref_s = LO.sync(Z.copy())
    assert np.array_equal(P.cpu().numpy().view(np.uint64), ref_p.view(np.uint64))
    assert np.array_equal(dZ.cpu().numpy().view(np.uint64), ref_s.view(np.uint64))


@pytest.mark.parametrize("name", sorted(MESHES))
def test_rk4_steps_vs_oracle(name, O):
    B, LV, spec, LO = setup(name, O)
    Z0 = LO.initial_data(eps=1e-8)
    m = B.Mesh(spec)
    # initial data per level grid on the GPU, then the level sync
    dI = torch.zeros((24, spec.n_nodes), dtype=torch.float64, device="cuda")
    LV.initial_data_levels(dI, spec, mesh=m)
    torch.cuda.synchronize()
    assert ol.rel_err(Z0, dI.cpu().numpy()).max() <= 1e-14
    dt = 0.25 * spec.h
    prm = B.default_params()
    for flags in (B.PLAN_ENFORCE_STAGES, B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH):
        Z = Z0.copy()
        dZ = dev(Z0)
        plan = B.RK4Plan(m, prm, flags)
        for _ in range(2):
            Z = LO.rk4_step(Z, dt, ol.params())
            plan.step(dZ, dt)
        torch.cuda.synchronize()
        assert plan.violations() == 0
        plan.close()
        got = dZ.cpu().numpy()
        err = ol.rel_err(Z, got)
        assert err.max() <= 1e-13, (err.max(), int(err.argmax()))
        for v in (0, 1, 2):  # the increments of alpha, chi, K
            d_ref, d_got = Z[v] - Z0[v], got[v] - Z0[v]
            assert np.abs(d_got - d_ref).max() <= 1e-10 * np.abs(d_ref).max(), v
        # levels agree where they coincide: the sync leaves no coarse node
        # under a finer box different from the fine node
        assert np.isfinite(got).all()


def test_transfer_bit_exact(O):
    """Transfer to a different hierarchy (one more level, a moved box) and
    to the same one (identity) against the oracle's transfer."""
    from oracle_levels import transfer as otransfer
    B, LV, spec, LO = setup("two", O)
    rng = np.random.default_rng(5)
    Z = LO.sync(rng.standard_normal((24, spec.n_nodes)))
    m = B.Mesh(spec)
    for boxes in ([((2, 2, 2), (4, 4, 4)), ((6, 6, 6), (4, 4, 4))], [((2, 2, 2), (4, 2, 4))],
                  list(MESHES["two"][1])):
        new = LV.generate_levels(spec.M0, boxes)
        nm = B.Mesh(new)
        dV = torch.empty((24, new.n_nodes), dtype=torch.float64, device="cuda")
        LV.transfer(m, dev(Z), nm, dV)
        ref = otransfer(LO, Z, LevelOracle(new, O))
        got = dV.cpu().numpy()
        assert np.array_equal(got.view(np.uint64), ref.view(np.uint64)), boxes
        if boxes == list(MESHES["two"][1]):
            assert np.array_equal(got.view(np.uint64), Z.view(np.uint64))
        nm.close()


def test_remesh_during_evolution(O):
    """Evolve, flag blocks with the exact wavelet test on the GPU (the 30 %
    with the largest score ratio), regrid, transfer and evolve on: the GPU
    against the oracle fed the same flags."""
    from oracle_levels import transfer as otransfer
    B, LV, spec, LO = setup("two", O)
    Z0 = LO.initial_data(eps=1e-8)
    m = B.Mesh(spec)
    dt = 0.25 * spec.h
    prm = B.default_params()
    dZ = dev(Z0)
    plan = B.RK4Plan(m, prm, B.PLAN_ENFORCE_STAGES)
    Z = Z0
    for _ in range(2):
        plan.step(dZ, dt)
        Z = LO.rk4_step(Z, dt, ol.params())
    P = torch.zeros((24, m.n_unzip), dtype=torch.float64, device="cuda")
    m.unzip(P, dZ)
    _, ratio, _ = B.wavelet_scores(m, P, tol=1e-6)
    r = ratio.cpu().numpy()
    flags = (r >= np.quantile(r, 0.7)).astype(np.uint8)
    new, nm, dV = LV.remesh(m, dZ, flags)
    assert new.nlevels >= 2
    LN = LevelOracle(new, O)
    V = otransfer(LO, Z, LN)
    assert ol.rel_err(V, dV.cpu().numpy()).max() <= 1e-13
    plan2 = B.RK4Plan(nm, prm, B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH)
    dt2 = 0.25 * new.h
    for _ in range(2):
        plan2.step(dV, dt2)
        V = LN.rk4_step(V, dt2, ol.params())
    torch.cuda.synchronize()
    assert plan.violations() == 0 and plan2.violations() == 0
    got = dV.cpu().numpy()
    assert np.isfinite(got).all()
    assert ol.rel_err(V, got).max() <= 1e-13


PATCHES = ((8, 4, 4), [(1, 0, (2, 2, 2), (4, 4, 4)), (1, 0, (10, 2, 2), (4, 4, 4)),
                       (2, 1, (6, 6, 6), (4, 4, 4))])


def test_patches_ghost_fill_sync_and_steps(O):
    """Two refined patches on level 1 (one refined again): ghost fill and
    sync bit-exact, two RK4 steps (graph) within 1e-13 of the oracle."""
    import bssn_b200 as B
    from bssn_b200 import levels as LV
    # origin off the node lattice of the punctures at (+-1, 0, 0), so no
    # node sits on a puncture (Brill-Lindquist data is singular there)
    spec = LV.generate_patches(*PATCHES, xmin=-8.25)
    LO = LevelOracle(spec, O)
    m = B.Mesh(spec)
    rng = np.random.default_rng(4)
    Z = rng.standard_normal((24, spec.n_nodes))
    P = torch.zeros((24, m.n_unzip), dtype=torch.float64, device="cuda")
    dZ = dev(Z)
    m.unzip(P, dZ)
    LV.sync(m, dZ)
    torch.cuda.synchronize()
    assert np.array_equal(P.cpu().numpy().view(np.uint64), LO.unzip(Z).view(np.uint64))
    assert np.array_equal(dZ.cpu().numpy().view(np.uint64), LO.sync(Z.copy()).view(np.uint64))
    Z0 = LO.initial_data(eps=1e-8)
    dt = 0.25 * spec.h
    dZ = dev(Z0)
    plan = B.RK4Plan(m, B.default_params(), B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH)
    Zr = Z0
    for _ in range(2):
        plan.step(dZ, dt)
        Zr = LO.rk4_step(Zr, dt, ol.params())
    torch.cuda.synchronize()
    assert plan.violations() == 0
    err = ol.rel_err(Zr, dZ.cpu().numpy())
    assert err.max() <= 1e-13, err.max()


def test_transfer_box_chain_to_patches(O):
    """Transfer from a box-per-level hierarchy to a two-patch one, bit-exact
    against the oracle's transfer."""
    from oracle_levels import transfer as otransfer
    import bssn_b200 as B
    from bssn_b200 import levels as LV
    old = LV.generate_levels((8, 4, 4), [((2, 2, 2), (12, 4, 4))])
    LOo = LevelOracle(old, O)
    Z = LOo.sync(np.random.default_rng(6).standard_normal((24, old.n_nodes)))
    new = LV.generate_patches(*PATCHES)
    mo, mn = B.Mesh(old), B.Mesh(new)
    dV = torch.empty((24, new.n_nodes), dtype=torch.float64, device="cuda")
    LV.transfer(mo, dev(Z), mn, dV)
    ref = otransfer(LOo, Z, LevelOracle(new, O))
    assert np.array_equal(dV.cpu().numpy().view(np.uint64), ref.view(np.uint64))


def test_remesh_into_patches_during_evolution(O):
    """Two refined patches evolve, the wavelet test flags blocks, the flags
    are clustered into new patches, the state is transferred and evolved on:
    the GPU against the oracle fed the same flags."""
    from oracle_levels import transfer as otransfer
    import bssn_b200 as B
    from bssn_b200 import levels as LV
    spec = LV.generate_patches((12, 4, 4), [(1, 0, (2, 2, 2), (4, 4, 4)), (1, 0, (16, 2, 2), (4, 4, 4))],
                               xmin=-8.25)
    LO = LevelOracle(spec, O)
    m = B.Mesh(spec)
    prm = B.default_params()
    dt = 0.25 * spec.h
    Z = LO.initial_data(eps=1e-8)
    dZ = dev(Z)
    plan = B.RK4Plan(m, prm, B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH)
    for _ in range(2):
        plan.step(dZ, dt)
        Z = LO.rk4_step(Z, dt, ol.params())
    P = torch.zeros((24, m.n_unzip), dtype=torch.float64, device="cuda")
    m.unzip(P, dZ)
    _, ratio, _ = B.wavelet_scores(m, P, tol=1e-6)
    r = ratio.cpu().numpy()
    flags = (r >= np.quantile(r, 0.7)).astype(np.uint8)
    new, nm, dV = LV.remesh(m, dZ, flags, patches=True)
    LN = LevelOracle(new, O)
    V = otransfer(LO, Z, LN)
    assert ol.rel_err(V, dV.cpu().numpy()).max() <= 1e-13
    plan2 = B.RK4Plan(nm, prm, B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH)
    dt2 = 0.25 * new.h
    for _ in range(2):
        plan2.step(dV, dt2)
        V = LN.rk4_step(V, dt2, ol.params())
    torch.cuda.synchronize()
    assert plan.violations() == 0 and plan2.violations() == 0
    got = dV.cpu().numpy()
    assert np.isfinite(got).all()
    # relative to each variable's largest magnitude: the noise-level
    # variables (|max| ~ 1e-6 on the finer patches) carry the rounding of
    # the FP64 right-hand side (1e-12 of them, ~1e-18 absolute)
    assert ol.rel_err(V, got).max() <= 1e-11


def test_learned_remesh_on_patch_mesh(O):
    """The learned remesh decision on a patch hierarchy: with every block
    deferred (lo = 0, hi = 1) it reproduces the exact wavelet test there;
    its flags drive a remesh into patches, and the evolution goes on."""
    import bssn_b200 as B
    from bssn_b200 import levels as LV
    spec = LV.generate_patches((12, 4, 4), [(1, 0, (2, 2, 2), (4, 4, 4)), (1, 0, (16, 2, 2), (4, 4, 4))],
                               xmin=-8.25)
    m = B.Mesh(spec)
    U = torch.zeros((24, spec.n_nodes), dtype=torch.float64, device="cuda")
    LV.initial_data_levels(U, spec, mesh=m)
    plan = B.RK4Plan(m, B.default_params(), B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH)
    plan.step(U, 0.25 * spec.h)
    P = torch.zeros((24, m.n_unzip), dtype=torch.float64, device="cuda")
    m.unzip(P, U)
    net = B.RemeshMLP(seed=6)
    net.lo, net.hi = 0.0, 1.0
    flags, stats = B.remesh_decide(m, P, net, tol=1e-6, audit_frac=0.05)
    _, _, exact = B.wavelet_scores(m, P, tol=1e-6)
    torch.cuda.synchronize()
    assert torch.equal(flags, exact)
    net.lo, net.hi = 0.02, 0.98
    flags, stats = B.remesh_decide(m, P, net, tol=1e-6, audit_frac=0.05)
    torch.cuda.synchronize()
    if int(flags.sum()) == 0:
        flags[0] = 1  # a decision that refines somewhere, to exercise the remesh
    new, nm, V = LV.remesh(m, U, flags, patches=True)
    plan2 = B.RK4Plan(nm, B.default_params(), B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH)
    plan2.step(V, 0.25 * new.h)
    torch.cuda.synchronize()
    assert bool(torch.isfinite(V).all()) and plan2.violations() == 0


@pytest.mark.parametrize("name", sorted(MESHES))
def test_constraints_on_level_mesh(name, O):
    """Hamiltonian and momentum constraints on a level mesh after one RK4
    step: every node owned by a zone carries the oracle's
    orc_physical_constraints (physcon.cpp:12-89 restated) of that zone's
    block, nodes filled from another level are 0 (within 1e-12 of each
    field's largest value, as the single-level constraint tests)."""
    import ctypes as C
    B, LV, spec, LO = setup(name, O)
    m = B.Mesh(spec)
    dZ = torch.zeros((24, spec.n_nodes), dtype=torch.float64, device="cuda")
    LV.initial_data_levels(dZ, spec, mesh=m)
    plan = B.RK4Plan(m, B.default_params(), B.PLAN_ENFORCE_STAGES | B.PLAN_GRAPH)
    plan.step(dZ, 0.25 * spec.h)
    P = torch.zeros((24, m.n_unzip), dtype=torch.float64, device="cuda")
    m.unzip(P, dZ)
    cons = torch.full((4, spec.n_nodes), np.nan, dtype=torch.float64, device="cuda")
    B.constraints(m, cons, P)
    torch.cuda.synchronize()
    plan.close()
    Uz = P.cpu().numpy()
    Cz = np.zeros((24, m.n_unzip))
    ws = np.zeros(288 * 55 ** 3)
    for b in range(spec.nblocks):
        blk = spec.blocks[b]
        s = int(blk.sz)
        pm, px = np.array(blk.ptmin[:]), np.array(blk.ptmax[:])
        O.lib.orc_physical_constraints(ol.rows(Cz), ol.rows(Uz), C.c_uint(int(blk.offset)), ol.P(pm), ol.P(px),
                                       (C.c_uint * 3)(s, s, s), C.c_uint(int(blk.bflag)), ol.P(ws))
    zs = LV.level_maps(spec)["zip_src"]
    own = zs >= 0
    ref = np.zeros((4, spec.n_nodes))
    ref[:, own] = Cz[:4, zs[own]]
    got = cons.cpu().numpy()
    assert np.isfinite(got).all()
    assert not got[:, ~own].any()
    err = ol.rel_err(ref, got)
    assert err.max() <= 1e-12, err


def test_full_evolution_driver_small():
    """The full-evolution driver on a small 3-level mesh: the exact run and
    the learned run (two networks trained on the exact run's refine and keep
    labels) both evolve 20 steps with a remesh test every 5, stay finite with
    no enforcement violation, and report four constraint-norm entries plus
    the final one, and the decision counters."""
    from bssn_b200 import evolve as EV
    res = EV.main(["--M0", "8", "--levels", "3", "--max-levels", "3", "--steps", "20", "--remesh-every", "5",
                   "--diag-every", "5", "--train-steps", "50"])
    for r in (res["exact"], res["learned"]):
        assert r["finite"] and r["violations"] == 0
        assert r["tests"] == 3 and len(r["history"]) == 5
        assert all(np.isfinite(h[2:]).all() and h[2] > 0 for h in map(np.asarray, r["history"]))
    assert res["exact"]["exact_refinements"] > 0 and res["exact"]["exact_keeps"] > 0
    assert res["compare"]["exact_refinements_learned_run"] > 0
