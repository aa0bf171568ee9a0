"""GPU tests of the remesh indicator: the exact wavelet test and the block
features against the CPU oracle, the BF16 MLP forward / backward / Adam
kernels against a float64 numpy restatement (same BF16-rounded weights), and
the learned decision against the exact test."""
import ctypes as C
import time

import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


@pytest.fixture(scope="module")
def B():
    import bssn_b200
    return bssn_b200


@pytest.fixture(scope="module")
def state(B):
    """A mixed mesh, evolved a few steps so the fields have structure."""
    spec = B.generate_mesh(1, (2, 1, 1), seed=1, xmin=-8.25)
    m = B.Mesh(spec)
    U = torch.zeros((24, spec.n_nodes), dtype=torch.float64, device="cuda")
    B.initial_data(U, spec, bh=(0.6, -4.1, -4.2, -0.6, -4.1, -4.2))
    plan = B.RK4Plan(m, B.default_params())
    for _ in range(3):
        plan.step(U, 0.25 * spec.h)
    Pz = torch.zeros((24, m.n_unzip), dtype=torch.float64, device="cuda")
    m.unzip(Pz, U)
    torch.cuda.synchronize()
    return spec, m, Pz


def test_wavelet_scores_vs_oracle(B, state):
    spec, m, Pz = state
    scores, ratio, flags = B.wavelet_scores(m, Pz, tol=1e-6)
    torch.cuda.synchronize()
    U = Pz.cpu().numpy()
    ne = B.lib.bssn_mesh_num_elements(m.h)
    ref = np.zeros(ne * 24)
    O = ol.oracle()
    O.lib.orc_wavelet_scores(ol.rows(U), spec.blocks, spec.nblocks, 24, ref.ctypes.data_as(ol._dp))
    got = scores.cpu().numpy().ravel()
    # identical per-node coefficients; partial-sum order identical too
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
    # per-block flags: any element / variable above tol
    first = np.cumsum([0] + [((int(s) - 7) // 6) ** 3 for s in spec.sides])
    rmax = np.array([ref.reshape(ne, 24)[first[b]:first[b + 1]].max() for b in range(spec.nblocks)])
    assert np.array_equal(flags.cpu().numpy(), (rmax / 1e-6 > 1.0).astype(np.uint8))


def test_block_features_vs_oracle(B, state):
    spec, m, Pz = state
    f = B.block_features(m, Pz).cpu().numpy()
    U = Pz.cpu().numpy()
    ref = np.zeros((spec.nblocks, 16), dtype=np.float32)
    ol.oracle().lib.orc_block_features(ol.rows(U), spec.blocks, spec.nblocks, ref.ctypes.data_as(C.c_void_p))
    assert np.allclose(f, ref, rtol=1e-6, atol=1e-6)


# ---- float64 numpy restatement of the network --------------------------------
def _split(p):
    return (p[0:1024].reshape(64, 16), p[1024:1088], p[1088:5184].reshape(64, 64), p[5184:5248],
            p[5248:5312], p[5312])


def _gelu(a):
    from scipy.special import erf
    return 0.5 * a * (1.0 + erf(a / np.sqrt(2.0)))


def _gelu_grad(a):
    from scipy.special import erf
    return 0.5 * (1.0 + erf(a / np.sqrt(2.0))) + a * np.exp(-0.5 * a * a) / np.sqrt(2 * np.pi)


def _np_forward_backward(p, norm, X, Y, Cw):
    W1, b1, W2, b2, W3, b3 = _split(p)
    x = (X - norm[:16]) * norm[16:]
    a1 = x @ W1.T + b1
    h1 = _gelu(a1)
    a2 = h1 @ W2.T + b2
    h2 = _gelu(a2)
    z = h2 @ W3 + b3
    n = len(X)
    loss = np.sum(Cw * (np.maximum(z, 0) - z * Y + np.log1p(np.exp(-np.abs(z))))) / n
    dz = Cw * (1 / (1 + np.exp(-z)) - Y) / n
    gW3 = h2.T @ dz
    gb3 = dz.sum()
    da2 = np.outer(dz, W3) * _gelu_grad(a2)
    gW2 = da2.T @ h1
    gb2 = da2.sum(0)
    da1 = (da2 @ W2) * _gelu_grad(a1)
    gW1 = da1.T @ x
    gb1 = da1.sum(0)
    g = np.concatenate([gW1.ravel(), gb1, gW2.ravel(), gb2, gW3, [gb3]])
    return z, loss, g


def test_mlp_forward_backward_vs_numpy(B):
    net = B.RemeshMLP(seed=3)
    rng = np.random.default_rng(0)
    n = 1000
    X = torch.tensor(rng.standard_normal((n, 16)) * 2 + 1, dtype=torch.float32, device="cuda")
    Y = torch.tensor((rng.random(n) < 0.3).astype(np.float32), device="cuda")
    Cw = torch.tensor(rng.uniform(0.5, 2.0, n).astype(np.float32), device="cuda")
    net.set_norm(X)
    z = net.logits_fp32(X)
    g, loss = net.grad(X, Y, Cw)
    torch.cuda.synchronize()
    p = net.wq.float().cpu().numpy().astype(np.float64)  # the BF16 values the kernels use
    norm = net.norm.cpu().numpy().astype(np.float64)
    zr, lr, gr = _np_forward_backward(p, norm, X.cpu().numpy().astype(np.float64), Y.cpu().numpy(),
                                      Cw.cpu().numpy())
    assert np.allclose(z.cpu().numpy(), zr, rtol=1e-4, atol=1e-4)
    assert abs(loss.item() - lr) <= 1e-5 * abs(lr)
    gg = g.cpu().numpy()
    assert np.abs(gg - gr).max() <= 1e-3 * np.abs(gr).max(), np.abs(gg - gr).max() / np.abs(gr).max()


def _bf16(a):
    """Round float32 values to BF16 (nearest, ties to even), as float32."""
    u = np.ascontiguousarray(a, dtype=np.float32).view(np.uint32).astype(np.uint64)
    u = ((u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000).astype(np.uint32)
    return u.view(np.float32)


def test_mlp_tensor_core_forward(B):
    """The decisions' forward on the tensor cores (mma.sync m16n8k16, BF16
    operands, FP32 accumulation) against a float64 restatement that rounds
    the normalised inputs and the hidden activations to BF16 as the operands
    do, and close to the FP32-activation forward; 1001 samples leave a
    partial last warp."""
    from scipy.special import erf
    net = B.RemeshMLP(seed=7)
    rng = np.random.default_rng(3)
    n = 1001
    X = torch.tensor(rng.standard_normal((n, 16)) * 2 + 1, dtype=torch.float32, device="cuda")
    net.set_norm(X)
    z = net.logits(X).cpu().numpy().astype(np.float64)
    z32 = net.logits_fp32(X).cpu().numpy().astype(np.float64)
    p = net.wq.float().cpu().numpy().astype(np.float64)
    norm = net.norm.cpu().numpy()
    W1, b1, W2, b2, W3, b3 = _split(p)
    gelu = lambda a: 0.5 * a * (1.0 + erf(a / np.sqrt(2.0)))
    x = _bf16((X.cpu().numpy() - norm[:16]) * norm[16:]).astype(np.float64)
    h1 = _bf16(gelu(x @ W1.T + b1)).astype(np.float64)
    zr = gelu(h1 @ W2.T + b2) @ W3 + b3
    scale = np.abs(zr).max()
    assert np.abs(z - zr).max() <= 5e-3 * scale, np.abs(z - zr).max() / scale
    assert np.abs(z - z32).max() <= 3e-2 * np.abs(z32).max(), np.abs(z - z32).max() / np.abs(z32).max()


def test_adam_step_vs_numpy(B):
    net = B.RemeshMLP(seed=4)
    rng = np.random.default_rng(1)
    g = torch.tensor(rng.standard_normal(B.MLP_NPARAM).astype(np.float32), device="cuda")
    p0 = net.master.cpu().numpy().astype(np.float64)
    net.step(g, lr=1e-2)
    torch.cuda.synchronize()
    gn = g.cpu().numpy().astype(np.float64)
    m = 0.1 * gn
    v = 0.001 * gn * gn
    ref = p0 - 1e-2 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
    assert np.allclose(net.master.cpu().numpy(), ref, rtol=1e-5, atol=1e-6)
    assert torch.equal(net.wq, net.master.to(torch.bfloat16))


def test_learned_decision_matches_exact_where_it_defers(B, state):
    """Blocks the network defers (uncertain or audited) get exactly the
    exact-test flag; with lo=0, hi=1 every block defers and the learned
    pipeline reproduces the exact test."""
    spec, m, Pz = state
    net = B.RemeshMLP(seed=5)
    net.lo, net.hi = 0.0, 1.0
    flags, stats = B.remesh_decide(m, Pz, net, tol=1e-6, audit_frac=0.05)
    _, _, exact = B.wavelet_scores(m, Pz, tol=1e-6)
    torch.cuda.synchronize()
    assert torch.equal(flags, exact)
    assert int(stats[0]) + int(stats[1]) == spec.nblocks


def test_decide2_matches_exact_where_it_defers(B, state):
    """The one-pass two-flag decision: with both networks unsure of every
    block (lo = 0, hi = 1) it reproduces the exact refine flags (score above
    tol) and keep flags (above 0.1 tol) on every block."""
    spec, m, Pz = state
    nr, nk = B.RemeshMLP(seed=5), B.RemeshMLP(seed=6)
    nr.lo, nr.hi, nk.lo, nk.hi = 0.0, 1.0, 0.0, 1.0
    refine, keep, stats = B.remesh_decide2(m, Pz, nr, nk, tol=1e-6, keep_fac=0.1, audit_frac=0.05)
    _, ratio, exact = B.wavelet_scores(m, Pz, tol=1e-6)
    torch.cuda.synchronize()
    assert torch.equal(refine, exact)
    assert torch.equal(keep, (ratio > 0.1).to(torch.uint8))
    st = stats.cpu().tolist()
    assert st[0] == spec.nblocks and st[1] == spec.nblocks and st[2] == 0
    assert st[4] == int(exact.sum()) and st[6] == int((ratio > 0.1).sum())


def test_decide2_partial_list_matches_exact(B, state):
    """The exact test on part of the mesh (the compacted element list of the
    deferred blocks): refine network unsure of every block, keep network
    sure (lo = hi = 0.5), so only the blocks the keep network would keep
    (p > 0.5) are deferred for refine; there the refine flag equals the
    exact test's, and elsewhere it is 0 or (audited blocks) the exact flag."""
    spec, m, Pz = state
    nr, nk = B.RemeshMLP(seed=5), B.RemeshMLP(seed=8)
    nr.lo, nr.hi, nk.lo, nk.hi = 0.0, 1.0, 0.5, 0.5
    f = B.block_features(m, Pz)
    nk.set_norm(f)
    # output bias at minus the median logit: about half the blocks deferred
    nk.master[B.MLP_NPARAM - 1] -= float(nk.logits(f).median())
    nk.wq = nk.master.to(torch.bfloat16)
    lk = nk.logits(f).cpu().numpy()
    refine, keep, stats = B.remesh_decide2(m, Pz, nr, nk, tol=1e-6, keep_fac=0.1, audit_frac=0.05)
    _, ratio, exact = B.wavelet_scores(m, Pz, tol=1e-6)
    torch.cuda.synchronize()
    r, e = refine.cpu().numpy(), exact.cpu().numpy()
    deferred = lk > 1e-3
    sure_no = lk < -1e-3
    assert 0 < deferred.sum() < spec.nblocks
    assert np.array_equal(r[deferred], e[deferred])
    assert np.all(r[sure_no] <= e[sure_no])
    assert stats.cpu().tolist()[0] == int((lk > 0).sum())


def test_decide2_nothing_deferred(B, state):
    """Both networks sure of every block (lo = hi = 0.5) and no audit: the
    exact test's element list is empty, and the flags are the networks'
    decisions with the refine-implies-keep rule."""
    spec, m, Pz = state
    nr, nk = B.RemeshMLP(seed=5), B.RemeshMLP(seed=8)
    f = B.block_features(m, Pz)
    nr.set_norm(f)
    nk.set_norm(f)
    nr.lo = nr.hi = nk.lo = nk.hi = 0.5
    refine, keep, stats = B.remesh_decide2(m, Pz, nr, nk, tol=1e-6, keep_fac=0.1, audit_frac=0.0)
    pr = torch.sigmoid(nr.logits(f)).cpu().numpy()
    pk = torch.sigmoid(nk.logits(f)).cpu().numpy()
    torch.cuda.synchronize()
    assert stats.cpu().tolist() == [0] * 8
    # away from the threshold, where host and device sigmoids cannot disagree
    sure = (np.abs(pr - 0.5) > 1e-4) & (np.abs(pk - 0.5) > 1e-4)
    want_r = (pr >= 0.5) & (pk > 0.5)
    want_k = (pk >= 0.5) | (pr >= 0.5)
    assert np.array_equal(refine.cpu().numpy()[sure], want_r[sure].astype(np.uint8))
    assert np.array_equal(keep.cpu().numpy()[sure], want_k[sure].astype(np.uint8))


def test_element_features_vs_oracle(B, state):
    spec, m, Pz = state
    f = B.element_features(m, Pz).cpu().numpy()
    U = Pz.cpu().numpy()
    ne = B.lib.bssn_mesh_num_elements(m.h)
    ref = np.zeros((ne, 16), dtype=np.float32)
    ol.oracle().lib.orc_element_features(ol.rows(U), spec.blocks, spec.nblocks, ref.ctypes.data_as(C.c_void_p))
    assert np.allclose(f, ref, rtol=1e-6, atol=1e-6)


def test_decide2_elem_defer_all_matches_exact(B, state):
    """Per-element decision with both networks unsure of every element: the
    exact test runs on every element and the block flags equal the exact
    test's block flags."""
    spec, m, Pz = state
    nr, nk = B.RemeshMLP(seed=5), B.RemeshMLP(seed=6)
    nr.lo, nr.hi, nk.lo, nk.hi = 0.0, 1.0, 0.0, 1.0
    refine, keep, stats = B.remesh_decide2_elem(m, Pz, nr, nk, tol=1e-6, keep_fac=0.1, audit_frac=0.05)
    _, ratio, exact = B.wavelet_scores(m, Pz, tol=1e-6)
    torch.cuda.synchronize()
    ne = B.lib.bssn_mesh_num_elements(m.h)
    assert torch.equal(refine, exact)
    assert torch.equal(keep, (ratio > 0.1).to(torch.uint8))
    st = stats.cpu().tolist()
    assert st[0] == ne and st[1] == ne and st[2] == 0


def test_decide2_elem_nothing_deferred(B, state):
    """Per-element decision with both networks sure everywhere and no audit:
    no element reaches the exact test, and a block takes a flag when any of
    its elements' network decisions does."""
    spec, m, Pz = state
    fe = B.element_features(m, Pz)
    nr, nk = B.RemeshMLP(seed=5), B.RemeshMLP(seed=8)
    nr.set_norm(fe)
    nk.set_norm(fe)
    nr.lo = nr.hi = nk.lo = nk.hi = 0.5
    refine, keep, stats = B.remesh_decide2_elem(m, Pz, nr, nk, tol=1e-6, keep_fac=0.1, audit_frac=0.0)
    pr = torch.sigmoid(nr.logits(fe)).cpu().numpy()
    pk = torch.sigmoid(nk.logits(fe)).cpu().numpy()
    torch.cuda.synchronize()
    assert stats.cpu().tolist() == [0] * 8
    er = (pr >= 0.5) & (pk > 0.5)
    ek = (pk >= 0.5) | (pr >= 0.5)
    sure = (np.abs(pr - 0.5) > 1e-4) & (np.abs(pk - 0.5) > 1e-4)
    first = np.cumsum([0] + [((int(s) - 7) // 6) ** 3 for s in spec.sides])
    r, k = refine.cpu().numpy(), keep.cpu().numpy()
    checked = 0
    for b in range(spec.nblocks):
        sl = slice(first[b], first[b + 1])
        if sure[sl].all():
            assert r[b] == int(er[sl].any()) and k[b] == int(ek[sl].any()), b
            checked += 1
    assert checked > spec.nblocks // 2


def test_decide2_elem_settled_blocks(B, state):
    """A block takes a flag when any of its elements does.  Keep network sure
    of every element (keep), refine network unsure: only the refine flag is
    open, every element goes to the exact test for it and the block refine
    flags equal the exact test's.  Refine network sure of every element:
    every block refines and keeps, and no element is deferred."""
    spec, m, Pz = state
    ne = B.lib.bssn_mesh_num_elements(m.h)
    nr, nk = B.RemeshMLP(seed=5), B.RemeshMLP(seed=8)
    _, _, exact = B.wavelet_scores(m, Pz, tol=1e-6)
    nr.lo, nr.hi, nk.lo, nk.hi = 0.0, 1.0, 0.0, 0.0
    refine, keep, stats = B.remesh_decide2_elem(m, Pz, nr, nk, tol=1e-6, keep_fac=0.1, audit_frac=0.05)
    torch.cuda.synchronize()
    assert torch.equal(refine, exact)
    assert bool((keep == 1).all())
    st = stats.cpu().tolist()
    assert st[0] == ne and st[1] == 0 and st[2] == 0
    nr.lo, nr.hi, nk.lo, nk.hi = 0.0, 0.0, 0.0, 1.0
    refine, keep, stats = B.remesh_decide2_elem(m, Pz, nr, nk, tol=1e-6, keep_fac=0.1, audit_frac=0.0)
    torch.cuda.synchronize()
    assert bool((refine == 1).all()) and bool((keep == 1).all())
    assert stats.cpu().tolist()[:3] == [0, 0, 0]


def test_trained_indicator_meets_the_contract(B):
    """Train on labels from small mixed-mesh runs; set the thresholds on a
    validation split with a margin of one logit unit; evaluate on blocks of
    runs with other seeds: the learned decision misses at most 0.1 % of the
    blocks the exact test refines there, and on a fresh config-2-sized
    snapshot (3,948 blocks) it is at least 5 times faster than the
    exact test on every block."""
    from bssn_b200 import remesh_train as rt
    X, Y = rt.collect(16000, dims=(4, 3, 3), log=lambda *a: None)
    assert 0.005 < Y.mean() < 0.9
    net = B.RemeshMLP(seed=0)
    rt.train(net, X[:12000], Y[:12000], steps=800, batch=4096, log=lambda *a: None)
    pv = torch.sigmoid(net.logits(torch.tensor(X[12000:], device="cuda"))).cpu().numpy()
    net.lo, net.hi = rt.pick_thresholds(pv, Y[12000:], fn_target=1e-3, margin=1.0)
    Xh, Yh = rt.collect(6000, dims=(4, 3, 3), seed0=500, log=lambda *a: None)
    ev = rt.evaluate(net, Xh, Yh)
    assert ev["positives"] > 200, ev
    assert ev["false_negative_rate"] <= 1e-3, ev
    assert ev["deferred_fraction"] < 0.3, ev
    tm = rt.time_decisions(net, dims=(7, 5, 4))
    assert tm["speedup"] >= 5.0, tm
    assert tm["missed_refinements"] <= max(1, tm["exact_refinements"] // 1000), tm
