"""GPU test of bssn_remesh_mlp_bwd_noalloc_bf16: the network-gradient entry
point for callers that cannot allocate device memory when they need a
gradient (an application that owns all device memory through its own pool,
a time-stepping loop that must not pay cudaMalloc's synchronisation, latency
or failure mid-run).  It must give the same
gradient and loss as the regular entry point, which works in caller-provided
scratch, on consecutive calls (the fixed device array it uses keeps the
previous call's contents), and must refuse batches above its fixed limit
without launching anything.  Collected last so a failure here cannot hide
the other tests' results."""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

LIMIT = 16384
BSSN_ELIMIT = 6


def _vp(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


@pytest.fixture(scope="module")
def lib():
    import bssn_b200 as B
    L = B.lib
    vp = C.c_void_p
    L.bssn_remesh_mlp_bwd_noalloc_bf16.argtypes = [vp, vp, vp, vp, vp, C.c_int, vp, vp, vp]
    L.bssn_remesh_mlp_bwd_noalloc_bf16.restype = C.c_int
    return L


def _inputs(n, seed):
    rng = np.random.default_rng(seed)
    X = torch.tensor(rng.standard_normal((n, 16)).astype(np.float32), device="cuda")
    Y = torch.tensor((rng.random(n) < 0.4).astype(np.float32), device="cuda")
    Cw = torch.tensor(rng.uniform(0.5, 2.0, n).astype(np.float32), device="cuda")
    return X, Y, Cw


def _regular(B, net, X, Y, Cw):
    g, loss = net.grad(X, Y, Cw)
    return g, loss


def _noalloc(lib, B, net, X, Y, Cw):
    g = torch.full((B.MLP_NPARAM,), float("nan"), dtype=torch.float32, device="cuda")
    loss = torch.full((1,), float("nan"), dtype=torch.float32, device="cuda")
    rc = lib.bssn_remesh_mlp_bwd_noalloc_bf16(_vp(net.wq), _vp(net.norm), _vp(X), _vp(Y), _vp(Cw),
                                              X.shape[0], _vp(g), _vp(loss), B.stream_ptr())
    assert rc == 0
    return g, loss


def test_noalloc_gradient_matches_regular_entry_point_twice(lib):
    import bssn_b200 as B
    net = B.RemeshMLP(seed=11)
    # different batches in a row: a later call must not see an earlier
    # call's partial sums; 3001 leaves a partial last CTA.  Both entry points
    # run the same kernels with the same part count and reduction order, so
    # the results must be bit-identical (a wrong part stride or loss-partial
    # offset would show in the low bits).
    for n, seed in ((LIMIT, 1), (3001, 2), (3001, 2)):
        X, Y, Cw = _inputs(n, seed)
        net.set_norm(X)
        g_ref, l_ref = _regular(B, net, X, Y, Cw)
        g, loss = _noalloc(lib, B, net, X, Y, Cw)
        torch.cuda.synchronize()
        assert torch.isfinite(g).all()
        assert torch.equal(g, g_ref)
        assert torch.equal(loss.reshape(-1), l_ref.reshape(-1))


def test_noalloc_rejects_batches_above_its_limit(lib):
    import bssn_b200 as B
    net = B.RemeshMLP(seed=12)
    X, Y, Cw = _inputs(LIMIT + 1, 3)
    g = torch.zeros(B.MLP_NPARAM, dtype=torch.float32, device="cuda")
    rc = lib.bssn_remesh_mlp_bwd_noalloc_bf16(_vp(net.wq), None, _vp(X), _vp(Y), _vp(Cw), LIMIT + 1,
                                              _vp(g), None, B.stream_ptr())
    assert rc == BSSN_ELIMIT
    torch.cuda.synchronize()
    assert not g.any()
