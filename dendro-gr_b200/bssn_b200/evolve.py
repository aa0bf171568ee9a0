"""Full evolution of a puncture pair with periodic remeshing, once with the
exact wavelet test deciding every remesh and once with the learned decision
(network + exact test on the uncertain band + seeded audit), on a
multi-level mesh.

The loop follows the reference's time loop (BSSN_GR/src/bssngr_main.cpp:
409-425): every `remesh_every` steps (BSSN_REMESH_TEST_FREQ, step != 0) the
refinement test runs on the unzipped state (BSSNCtx::is_remesh,
BSSN_GR/src/bssnCtx.cpp:1184-1230, which calls isReMeshWAMR); when the grid
it asks for differs from the current one the mesh is rebuilt and the state
carried over (remesh_and_gridtransfer), and the evolution goes on.  Here the
grid is a box-per-level hierarchy (levels.regrid_boxes), the transfer is
levels.transfer, and each RK4 step is the graph-replayed plan.

Each test gives two flags per block, as the reference's does (BSSN_GR/src/
dataUtils.cpp:413-480): refine (wavelet score above tol) and keep (score
above BSSN_DENDRO_AMR_FAC * tol, 0.1 in BSSN_GR/pars/q1.par.json: the block
holds its level; below it the block may coarsen).  Without that hysteresis
a refined region scores below tol on its finer grid, coarsens at the next
test and refines again at the one after.

The learned run uses two networks of the same shape, one per threshold,
trained on the labels the exact test gave during the exact run: features of
every element (the default) or every block at every remesh test.  Their
decision thresholds are set on the samples of the exact run's last fifth of
remesh tests, which the networks never saw in training (snapshots later in
the evolution, on the meshes of that time), and lowered by a margin in logit
units.  One decision pass serves both flags (bssn_remesh_decide2_elem_f64,
or bssn_remesh_decide2_f64 per block): the features once, both networks, and
one exact-test pass on the elements (blocks) either network is unsure of plus
a seeded audit sample; per element, a block takes a flag when any of its
elements does, so an uncertain corner of a large block no longer sends the
whole block to the exact test.  In the learned run the exact test is also
evaluated at every remesh test, outside the timed decision, to count the
refine and keep flags the decision missed.

    python -m bssn_b200.evolve --steps 1000 --remesh-every 10 --out run.json
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import (Mesh, NVARS, PLAN_ENFORCE_STAGES, PLAN_GRAPH, RemeshMLP, RK4Plan, block_features,
               constraints, default_params, element_features, remesh_decide2, remesh_decide2_elem,
               wavelet_scores)
from . import levels as LV
from .remesh_train import pick_thresholds, train

BH = (4.0, 0.0, 0.0, -4.0, 0.0, 0.0)   # punctures m = 0.5 at (+-4, 0, 0): separation 8


def nested_boxes(M0, nlevels):
    """Boxes of levels 1..nlevels-1, each M0 of its own octants per axis and
    centred on the origin (the middle half of its parent box)."""
    boxes, lo = [], 0
    for _ in range(1, nlevels):
        lo = 2 * lo + M0 // 2
        boxes.append(((lo,) * 3, (M0,) * 3))
    return boxes


def needs_remesh(cur, new):
    """Whether a regrid result asks for a new hierarchy: a level added or
    dropped, a box reaching outside the current one (refinement needed
    there), or a current box more than twice the volume asked for (room to
    coarsen).  Small shifts of the boxes keep the current mesh, so the grid
    does not change at every test."""
    if len(cur) != len(new):
        return True
    for (clo, cn), (nlo, nn) in zip(cur, new):
        clo, cn, nlo, nn = (np.asarray(x) for x in (clo, cn, nlo, nn))
        if np.any(nlo < clo) or np.any(nlo + nn > clo + cn) or np.prod(cn) > 2 * np.prod(nn):
            return True
    return False


def zones(spec):
    """Block-interior points of a mesh (the unit of a zone-update)."""
    return float(((np.asarray(spec.sides, dtype=np.float64) - 6.0) ** 3).sum())


def norm_mask(spec, bh=BH, radii=(0.5, 0.5), device="cpu"):
    """Boolean mask over the zipped nodes of a level mesh: the nodes a zone
    owns, outside the puncture radii.  Those are the independent points, each
    once on the finest grid that holds it; coarse nodes under a finer patch
    and patch-boundary nodes are filled from another level (the hanging
    nodes of the reference's octree are not unique nodes either)."""
    import torch
    own = torch.from_numpy(LV.level_maps(spec)["zip_src"] >= 0).to(device)
    far = torch.empty(spec.n_nodes, dtype=torch.bool, device=device)
    for g in spec.grids():
        nx, ny, nz = g["dims"]
        ax = [torch.arange(n, dtype=torch.float64, device=device) * g["h"] + g["origin"][d]
              for d, n in enumerate((nx, ny, nz))]
        z, y, x = ax[2][:, None, None], ax[1][None, :, None], ax[0][None, None, :]
        d1 = ((x - bh[0]) ** 2 + (y - bh[1]) ** 2 + (z - bh[2]) ** 2).sqrt()
        d2 = ((x - bh[3]) ** 2 + (y - bh[4]) ** 2 + (z - bh[5]) ** 2).sqrt()
        far[g["offset"]:g["offset"] + nx * ny * nz] = ((d1 >= radii[0]) & (d2 >= radii[1])).reshape(-1)
    return own & far


def level_norms(cons, mask):
    """Masked L2 norms sqrt(sum c^2 / N) of the 4 zipped constraint fields
    over the nodes of `mask` (computeConstraintL2Norm, BSSN_GR/include/
    grUtils.tcc:36-134, over unique points outside the puncture radii)."""
    c = cons[:, mask]
    return (c * c).mean(dim=1).sqrt().cpu().numpy().tolist()


class _State:
    """Mesh, plan and per-mesh buffers of one run."""

    def __init__(self, spec, mesh, U, params):
        import torch
        self.spec, self.mesh, self.U = spec, mesh, U
        torch.cuda.empty_cache()  # the library allocates beside torch's cache
        self.plan = RK4Plan(mesh, params, PLAN_ENFORCE_STAGES | PLAN_GRAPH)
        self.P = torch.empty((NVARS, mesh.n_unzip), dtype=torch.float64, device="cuda")
        self.cons = torch.zeros((4, spec.n_nodes), dtype=torch.float64, device="cuda")
        self.mask = None
        self.zones = zones(spec)

    def close(self):
        self.plan.close()
        self.mesh.close()


def run(indicator, a, nets=None, collect=False, log=print):
    """One evolution; indicator "exact" or "learned" (nets = the refine and
    keep networks).  Returns the run's record (and the collected features,
    refine and keep labels when collect)."""
    import torch
    params = default_params()
    spec = LV.generate_levels((a.M0,) * 3, nested_boxes(a.M0, a.levels), xmin=-a.half, L=2 * a.half,
                              max_w=a.max_block_octants)
    mesh = Mesh(spec)
    U = torch.zeros((NVARS, spec.n_nodes), dtype=torch.float64, device="cuda")
    LV.initial_data_levels(U, spec, mesh=mesh, bh=BH)
    st = _State(spec, mesh, U, params)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    rec = dict(indicator=indicator, evolve_ms=0.0, decide_ms=0.0, regrid_s=0.0, zone_updates=0.0,
               tests=0, remeshes=0, history=[], blocks=[spec.nblocks], levels=[spec.nlevels],
               missed=0, exact_refinements=0, keep_missed=0, exact_keeps=0,
               decide_stats=[0] * 8)
    X, Y, K = [], [], []
    t, step = 0.0, 0
    torch.cuda.synchronize()
    wall0 = time.perf_counter()

    def norms():
        st.mesh.unzip(st.P, st.U)
        constraints(st.mesh, st.cons, st.P)
        if st.mask is None:
            st.mask = norm_mask(st.spec, device="cuda")
        return level_norms(st.cons, st.mask)

    while True:
        if step % a.diag_every == 0 or step == a.steps:
            rec["history"].append([step, t] + norms())
        if step == a.steps:
            break
        if step > 0 and step % a.remesh_every == 0:
            st.mesh.unzip(st.P, st.U)
            e0.record()
            if indicator == "exact":
                scores, ratio, flags = wavelet_scores(st.mesh, st.P, tol=a.tol)
                keep = (ratio > a.amr_fac).to(torch.uint8)
            else:
                decide = remesh_decide2_elem if a.granularity == "element" else remesh_decide2
                flags, keep, stats = decide(st.mesh, st.P, nets[0], nets[1], tol=a.tol,
                                            keep_fac=a.amr_fac, audit_frac=a.audit, seed=step)
            e1.record()
            e1.synchronize()
            rec["decide_ms"] += e0.elapsed_time(e1)
            rec["tests"] += 1
            if indicator == "learned":
                _, ratio, exact = wavelet_scores(st.mesh, st.P, tol=a.tol)
                ekeep = ratio > a.amr_fac
                rec["missed"] += int(((flags == 0) & (exact == 1)).sum())
                rec["exact_refinements"] += int(exact.sum())
                rec["keep_missed"] += int(((keep == 0) & ekeep).sum())
                rec["exact_keeps"] += int(ekeep.sum())
                rec["decide_stats"] = [x + y for x, y in zip(rec["decide_stats"], stats.cpu().tolist())]
            else:
                rec["exact_refinements"] += int(flags.sum())
                rec["exact_keeps"] += int(keep.sum())
            if collect and a.granularity == "element":
                # per element: its largest score over the variables against
                # tol and amr_fac * tol (the block test's ratio, per element)
                r = scores.amax(dim=1) / a.tol
                X.append(element_features(st.mesh, st.P).cpu().numpy())
                Y.append((r > 1.0).float().cpu().numpy())
                K.append((r > a.amr_fac).float().cpu().numpy())
            elif collect:
                X.append(block_features(st.mesh, st.P).cpu().numpy())
                Y.append(flags.float().cpu().numpy())
                K.append(keep.float().cpu().numpy())
            f, k = flags.cpu().numpy(), keep.cpu().numpy()
            new_boxes = LV.regrid_boxes(st.spec, f, max_levels=a.max_levels, keep=k, max_n=a.max_box)
            if needs_remesh(st.spec.boxes[1:], new_boxes):
                w0 = time.perf_counter()
                st.P = st.cons = st.mask = None
                torch.cuda.empty_cache()
                spec2, mesh2, U2 = LV.remesh(st.mesh, st.U, f, max_levels=a.max_levels, keep=k, max_n=a.max_box)
                st.close()
                st = _State(spec2, mesh2, U2, params)
                torch.cuda.synchronize()
                rec["regrid_s"] += time.perf_counter() - w0
                rec["remeshes"] += 1
                rec["blocks"].append(spec2.nblocks)
                rec["levels"].append(spec2.nlevels)
                log(f"[{indicator}] step {step}: remesh -> {spec2.nblocks} blocks, {spec2.nlevels} levels")
        dt = a.cfl * st.spec.h
        n = min(a.steps - step, a.remesh_every - step % a.remesh_every, a.diag_every - step % a.diag_every)
        e0.record()
        for _ in range(n):
            st.plan.step(st.U, dt)
        e1.record()
        e1.synchronize()
        rec["evolve_ms"] += e0.elapsed_time(e1)
        rec["zone_updates"] += st.zones * n
        step += n
        t += n * dt
    torch.cuda.synchronize()
    rec["wall_s"] = time.perf_counter() - wall0
    rec["violations"] = st.plan.violations()
    rec["finite"] = bool(torch.isfinite(st.U).all())
    rec["zone_updates_per_s"] = rec["zone_updates"] / (rec["evolve_ms"] * 1e-3)
    log(f"[{indicator}] done: {rec['wall_s']:.1f} s, {rec['remeshes']} remeshes, "
        f"{rec['zone_updates_per_s'] / 1e6:.1f} M zone-updates/s")
    st.close()
    del st
    torch.cuda.empty_cache()
    if collect:
        return rec, np.concatenate(X), np.concatenate(Y), np.concatenate(K)
    return rec


def compare(ex, le):
    """Decision speed-up, missed refinements and the largest relative
    difference between the two constraint-norm histories."""
    h1 = np.asarray(ex["history"])[:, 2:]
    h2 = np.asarray(le["history"])[:, 2:]
    k = min(len(h1), len(h2))
    rel = np.abs(h1[:k] - h2[:k]) / np.maximum(np.abs(h1[:k]), 1e-300)
    return {"decision_speedup": ex["decide_ms"] / max(le["decide_ms"], 1e-9),
            "missed_refinements": le["missed"], "exact_refinements_learned_run": le["exact_refinements"],
            "false_negative_rate": le["missed"] / max(le["exact_refinements"], 1),
            "missed_keeps": le["keep_missed"], "exact_keeps_learned_run": le["exact_keeps"],
            "keep_false_negative_rate": le["keep_missed"] / max(le["exact_keeps"], 1),
            "norm_history_max_rel_diff": [float(x) for x in rel.max(axis=0)],
            "wall_ratio": ex["wall_s"] / le["wall_s"]}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--M0", type=int, default=24, help="level-0 octants per axis")
    ap.add_argument("--levels", type=int, default=7)
    ap.add_argument("--max-levels", type=int, default=7)
    ap.add_argument("--half", type=float, default=400.0, help="domain [-half, half]^3")
    ap.add_argument("--max-box", type=int, default=None, help="octants per axis and level (default M0)")
    ap.add_argument("--max-block-octants", type=int, default=8, choices=(1, 2, 4, 8),
                    help="largest block in octants per axis (1: every block 13^3; M0 20 with 7 levels "
                         "then gives 50,000 blocks)")
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--remesh-every", type=int, default=10)
    ap.add_argument("--diag-every", type=int, default=10)
    ap.add_argument("--cfl", type=float, default=0.25)
    ap.add_argument("--tol", type=float, default=1e-6)
    ap.add_argument("--amr-fac", type=float, default=0.1, help="keep threshold / tol (BSSN_DENDRO_AMR_FAC)")
    ap.add_argument("--audit", type=float, default=0.05)
    ap.add_argument("--train-steps", type=int, default=2000)
    ap.add_argument("--margin", type=float, default=0.5,
                    help="lower threshold margin in logit units (remesh_train.pick_thresholds)")
    ap.add_argument("--fp-target", type=float, default=1e-2,
                    help="fraction of validation negatives the upper threshold may let through "
                         "(extra refinement or a delayed coarsening, never a missed refinement)")
    ap.add_argument("--fn-target", type=float, default=1e-3,
                    help="missed-refinement budget of the refine network's lower threshold (half of it, "
                         "before the margin, on the validation samples)")
    ap.add_argument("--fn-keep", type=float, default=1e-2,
                    help="the same budget for the keep network (a missed keep lets a block coarsen one "
                         "test early; it never drops a refinement)")
    ap.add_argument("--granularity", default="element", choices=("element", "block"),
                    help="what the networks decide: each element (the exact test then runs on the "
                         "uncertain elements only) or each block")
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    a.max_box = a.max_box or a.M0
    import torch
    ex, X, Y, K = run("exact", a, collect=True)
    print(json.dumps({k: v for k, v in ex.items() if k != "history"}), flush=True)
    t0 = time.perf_counter()
    # samples in test order: train on the first four fifths of the tests,
    # thresholds on the last fifth (later snapshots, unseen in training)
    nva = max(len(X) // 5, 1)
    tr, va = np.arange(len(X) - nva), np.arange(len(X) - nva, len(X))
    nets = []
    for seed, lab in ((0, Y), (1, K)):
        net = RemeshMLP(seed=seed)
        train(net, X[tr], lab[tr], steps=a.train_steps, log=lambda s: None)
        pv = torch.sigmoid(net.logits(torch.tensor(X[va], device="cuda"))).cpu().numpy()
        fn = a.fn_target if seed == 0 else a.fn_keep
        net.lo, net.hi = pick_thresholds(pv, lab[va], fn_target=fn, fp_target=a.fp_target, margin=a.margin)
        nets.append(net)
    train_s = time.perf_counter() - t0
    le = run("learned", a, nets=nets)
    res = {"config": {k: getattr(a, k) for k in ("M0", "levels", "max_levels", "half", "max_box", "steps", "remesh_every",
                                                 "diag_every", "cfl", "tol", "amr_fac", "audit", "train_steps",
                                                 "margin", "fp_target", "fn_target", "fn_keep", "max_block_octants",
                                                 "granularity")},
           "training": {"samples": int(len(tr)), "validation": int(nva), "refine_labels": int(Y.sum()),
                        "keep_labels": int(K.sum()), "thresholds": [[n.lo, n.hi] for n in nets],
                        "seconds": train_s},
           "exact": ex, "learned": le, "compare": compare(ex, le)}
    print(json.dumps({k: v for k, v in res.items() if k not in ("exact", "learned")}))
    print(json.dumps({k: v for k, v in le.items() if k != "history"}))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)
    return res


if __name__ == "__main__":
    main()
