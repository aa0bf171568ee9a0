"""Training and evaluation of the learned remesh indicator.

Samples come from evolutions of seeded mixed-size meshes: at each snapshot
every block contributes its 16 features (bssn_remesh_features_f64) and the
label the exact wavelet test gives it (bssn_remesh_wavelet_f64).  The
network (BF16 compute, FP32 accumulation, Adam on FP32 masters) is trained
with the library's own forward / backward / Adam kernels; the decision
thresholds are then set on a validation split so that the blocks the
network alone would keep unrefined miss at most a target fraction of the
blocks the exact test refines; the uncertain band and a seeded audit sample
go to the exact test.

    python -m bssn_b200.remesh_train --samples 200000 --holdout 20000
"""
from __future__ import annotations

import argparse
import json
import time

import numpy as np

from . import (Mesh, RK4Plan, RemeshMLP, block_features, default_params, generate_mesh,
               initial_data, remesh_decide, wavelet_scores, NVARS)


def collect(n_samples, dims=(7, 5, 4), tol=1e-6, steps_between=4, seed0=100, log=print):
    """Features and exact labels from config-2 style runs (about 4,000 blocks
    per snapshot), puncture positions drawn by seed per run."""
    import torch
    X, Y = [], []
    have = 0
    run = 0
    while have < n_samples:
        rng = np.random.default_rng(seed0 + run)
        spec = generate_mesh(1, dims, seed=seed0 + run)
        m = Mesh(spec)
        U = torch.zeros((NVARS, spec.n_nodes), dtype=torch.float64, device="cuda")
        # punctures near the centre of the box, separation and offset by seed
        sep = rng.uniform(0.5, 2.0)
        c = np.array([rng.uniform(-1, 1), rng.uniform(-3, 1), rng.uniform(-3, -1)])
        bh = (c[0] + sep / 2, c[1], c[2], c[0] - sep / 2, c[1], c[2])
        initial_data(U, spec, bh=bh, seed=20261203 + run)
        plan = RK4Plan(m, default_params())
        Pz = torch.zeros((NVARS, m.n_unzip), dtype=torch.float64, device="cuda")
        for snap in range(5):
            m.unzip(Pz, U)
            f = block_features(m, Pz)
            _, ratio, flags = wavelet_scores(m, Pz, tol=tol)
            X.append(f.cpu().numpy())
            Y.append(flags.cpu().numpy().astype(np.float32))
            have += spec.nblocks
            for _ in range(steps_between):
                plan.step(U, 0.25 * spec.h)
        plan.close()
        del Pz, U
        m.close()
        log(f"run {run}: {have} samples, positive fraction {np.concatenate(Y).mean():.4f}")
        run += 1
    return np.concatenate(X)[:n_samples], np.concatenate(Y)[:n_samples]


def train(net: RemeshMLP, X, Y, steps=3000, batch=16384, lr=3e-3, seed=0, log=print):
    import torch
    Xd = torch.tensor(X, device="cuda")
    Yd = torch.tensor(Y, device="cuda")
    net.set_norm(Xd)
    pos = float(Y.mean())
    # balance the classes: positives weighted by (1-pos)/pos
    w = np.where(Y > 0.5, (1 - pos) / max(pos, 1e-6), 1.0).astype(np.float32)
    Wd = torch.tensor(w, device="cuda")
    g = torch.Generator(device="cuda").manual_seed(seed)
    n = len(X)
    for it in range(steps):
        idx = torch.randint(0, n, (min(batch, n),), device="cuda", generator=g)
        grad, loss = net.grad(Xd[idx].contiguous(), Yd[idx].contiguous(), Wd[idx].contiguous())
        net.step(grad, lr=lr * (0.5 * (1 + np.cos(np.pi * it / steps))))
        if it % 500 == 0 or it == steps - 1:
            log(f"step {it}: loss {loss.item():.5f}")
    return net


def pick_thresholds(p, y, fn_target=1e-3, fp_target=1e-3, margin=1.0):
    """lo: the largest threshold with (positives at p <= lo) / positives <=
    fn_target / 2 (half the budget, for margin), then lowered by `margin` in
    logit units (margin > 0 keeps room for snapshots unlike the validation
    ones: each unit widens the deferred band toward p = 0 by a factor of
    about e); hi: the smallest with (negatives at p >= hi) / negatives <=
    fp_target."""
    pos = p[y > 0.5]
    neg = p[y < 0.5]
    lo = float(np.quantile(pos, fn_target / 2, method="lower")) if len(pos) else 0.5
    if margin > 0 and 0.0 < lo < 1.0:
        z = np.log(lo / (1.0 - lo)) - margin
        lo = float(1.0 / (1.0 + np.exp(-z)))
    lo = np.nextafter(np.float32(lo), np.float32(0)).item()
    hi = float(np.quantile(neg, 1 - fp_target, method="higher")) if len(neg) else 0.5
    hi = np.nextafter(np.float32(hi), np.float32(1)).item()
    return lo, max(hi, lo)


def evaluate(net: RemeshMLP, X, Y):
    import torch
    p = torch.sigmoid(net.logits(torch.tensor(X, device="cuda"))).cpu().numpy()
    y = Y > 0.5
    pred = p >= 0.5
    tp = int((pred & y).sum())
    fp = int((pred & ~y).sum())
    fn = int((~pred & y).sum())
    kept = p <= net.lo           # network alone says "no refine"
    refined = p >= net.hi
    deferred = ~(kept | refined)
    system_fn = int((kept & y).sum())
    return {"n": int(len(y)), "positives": int(y.sum()),
            "precision@0.5": tp / max(tp + fp, 1), "recall@0.5": tp / max(tp + fn, 1),
            "lo": net.lo, "hi": net.hi, "deferred_fraction": float(deferred.mean()),
            "false_negatives": system_fn, "false_negative_rate": system_fn / max(int(y.sum()), 1),
            "false_positive_rate": float((refined & ~y).sum() / max(int((~y).sum()), 1))}


def time_decisions(net: RemeshMLP, dims=(7, 5, 4), seed=999, tol=1e-6, reps=5):
    """Remesh decision time on one config-2 style snapshot: the exact test
    on every block against the learned pipeline (features, network, exact
    test on the deferred and audited blocks), CUDA events, best of reps."""
    import torch
    spec = generate_mesh(1, dims, seed=seed)
    m = Mesh(spec)
    U = torch.zeros((NVARS, spec.n_nodes), dtype=torch.float64, device="cuda")
    initial_data(U, spec, bh=(0.5, -1.0, -2.0, -0.5, -1.0, -2.0))
    Pz = torch.zeros((NVARS, m.n_unzip), dtype=torch.float64, device="cuda")
    m.unzip(Pz, U)

    def best(fn):
        t = []
        for _ in range(reps + 1):
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record()
            out = fn()
            b.record()
            torch.cuda.synchronize()
            t.append(a.elapsed_time(b))
        return min(t[1:]), out
    t_exact, (_, _, exact) = best(lambda: wavelet_scores(m, Pz, tol=tol))
    t_learn, (flags, stats) = best(lambda: remesh_decide(m, Pz, net, tol=tol))
    st = stats.cpu().numpy().tolist()
    agree = bool(torch.equal(flags, exact))
    miss = int(((flags == 0) & (exact == 1)).sum())
    return {"blocks": spec.nblocks, "exact_ms": t_exact, "learned_ms": t_learn,
            "speedup": t_exact / t_learn, "stats": st, "flags_equal_exact": agree,
            "missed_refinements": miss, "exact_refinements": int(exact.sum())}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--samples", type=int, default=200000)
    ap.add_argument("--holdout", type=int, default=20000)
    ap.add_argument("--steps", type=int, default=3000)
    ap.add_argument("--out", default=None)
    a = ap.parse_args()
    t0 = time.time()
    X, Y = collect(a.samples + a.holdout + a.holdout)
    tr = slice(0, a.samples)
    va = slice(a.samples, a.samples + a.holdout)
    te = slice(a.samples + a.holdout, None)
    net = RemeshMLP(seed=0)
    train(net, X[tr], Y[tr], steps=a.steps)
    import torch
    pv = torch.sigmoid(net.logits(torch.tensor(X[va], device="cuda"))).cpu().numpy()
    net.lo, net.hi = pick_thresholds(pv, Y[va])
    res = {"train": evaluate(net, X[tr], Y[tr]), "heldout": evaluate(net, X[te], Y[te]),
           "timing": time_decisions(net), "wall_s": time.time() - t0}
    print(json.dumps(res))
    if a.out:
        with open(a.out, "w") as f:
            json.dump(res, f, indent=1)


if __name__ == "__main__":
    main()
