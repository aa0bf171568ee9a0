"""CPU tests: the oracle (this repository's CPU restatement) pinned against
the reference's own compiled arithmetic and against the committed golden
fixtures generated from it."""
import json
import os

import numpy as np
import pytest

import oracle_lib as ol

HERE = os.path.dirname(os.path.abspath(__file__))
GOLD = os.path.join(HERE, "golden", "rhs_golden.json")


@pytest.fixture(scope="module")
def O():
    return ol.oracle()


@pytest.fixture(scope="module")
def REF():
    r = ol.reference()
    if r is None:
        pytest.skip("oracle/_ref/libbssn_ref.so not built (reference tree absent)")
    return r


@pytest.mark.parametrize("side", [13, 19])
def test_stencils_bit_exact_vs_reference(O, REF, side):
    rng = np.random.default_rng(side)
    u = 1.0 + 1e-8 * rng.standard_normal(side ** 3)   # O(1) mean, tiny noise
    for kind in range(9):
        for bflag in range(64):
            a = REF.stencil(kind, u, 0.21, (side, side, side), bflag)
            b = O.stencil(kind, u, 0.21, (side, side, side), bflag)
            assert np.array_equal(a.view(np.uint64), b.view(np.uint64)), (kind, bflag)


def _load_golden():
    with open(GOLD) as f:
        return json.load(f)["cases"]


@pytest.mark.parametrize("ci", range(5))
def test_rhs_vs_golden(O, ci):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden as mg
    c = _load_golden()[ci]
    U, pmin, pmax = mg.golden_input(c["side"], c["h"], tuple(c["shift"]), c["noise"], c["seed"])
    R = O.bssnrhs(U, 0, pmin, pmax, c["side"], c["bflag"], ol.params())
    Ri = mg.interior(R, c["side"])
    for v in range(24):
        mx = float.fromhex(c["maxnorm"][v])
        got_mx = np.abs(Ri[v]).max()
        assert abs(got_mx - mx) <= 1e-12 * mx, (v, got_mx, mx)
        l2 = float.fromhex(c["l2"][v])
        assert abs(np.sqrt((Ri[v] ** 2).sum()) - l2) <= 1e-12 * l2, v
        for p, hv in zip(c["points"], c["values"][v]):
            ref = float.fromhex(hv)
            assert abs(R[v, p] - ref) <= 1e-12 * mx, (v, p)


@pytest.mark.parametrize("side,bflag", [(13, 0), (13, 63), (19, 21), (31, 42)])
def test_rhs_vs_reference_live(O, REF, side, bflag):
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden as mg
    U, pmin, pmax = mg.golden_input(side, 2.0 / (side - 7), (0.1, -1.1, -0.95), 1e-8, side + bflag)
    a = mg.interior(REF.bssnrhs(U, 0, pmin, pmax, side, bflag, ol.params()), side)
    b = mg.interior(O.bssnrhs(U, 0, pmin, pmax, side, bflag, ol.params()), side)
    err = ol.rel_err(a, b)
    assert err.max() <= 1e-12, (err.max(), int(err.argmax()))


@pytest.mark.parametrize("pset", ["eta_r", "cako_lambda"])
@pytest.mark.parametrize("side,bflag", [(13, 63), (19, 0)])
def test_rhs_vs_reference_live_params(O, REF, pset, side, bflag):
    """The restated right-hand side against the reference's generated
    equations with r-dependent eta, CAKO and other gauge parameters."""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden as mg
    prm = ol.params(**ol.PARAM_SETS[pset])
    U, pmin, pmax = mg.golden_input(side, 2.0 / (side - 7), (0.1, -1.1, -0.95), 1e-8, side + bflag)
    a = mg.interior(REF.bssnrhs(U, 0, pmin, pmax, side, bflag, prm), side)
    b = mg.interior(O.bssnrhs(U, 0, pmin, pmax, side, bflag, prm), side)
    err = ol.rel_err(a, b)
    assert err.max() <= 1e-12, (err.max(), int(err.argmax()))


def test_flat_space_rhs_is_zero(O):
    side = 13
    U = np.zeros((24, side ** 3))
    U[[0, 1, 12, 15, 17]] = 1.0
    pmin = np.array([2.0, 2.0, 2.0])
    R = O.bssnrhs(U, 0, pmin, pmin + 12 * 0.1, side, 0, ol.params())
    assert np.abs(R).max() == 0.0


def test_enforce_invariants(O):
    rng = np.random.default_rng(0)
    n = 1000
    Z = np.zeros((24, n))
    Z[[12, 15, 17]] = 1.0
    Z += 1e-3 * rng.standard_normal(Z.shape)
    Z[[0, 1]] = rng.uniform(1e-6, 1.0, (2, n))
    O.lib.orc_enforce.restype = ol.C.c_int64
    bad = O.lib.orc_enforce(ol.rows(Z), ol.C.c_int64(n), ol.C.c_double(1e-4))
    assert bad == 0
    g = Z[12:18]
    det = g[0] * (g[3] * g[5] - g[4] ** 2) - g[1] ** 2 * g[5] + 2 * g[1] * g[2] * g[4] - g[2] ** 2 * g[3]
    assert np.abs(det - 1).max() < 1e-6
    assert Z[0].min() >= 1e-4 and Z[1].min() >= 1e-4


@pytest.mark.parametrize("side,bflag", [(13, 0), (19, 63), (31, 21)])
def test_constraints_vs_reference_live(O, REF, side, bflag):
    """Hamiltonian / momentum constraints of the restatement against the
    reference's own physconeqs.cpp (physcon.cpp:12-89 control flow)."""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden as mg
    U, pmin, pmax = mg.golden_input(side, 2.0 / (side - 7), (0.1, -1.1, -0.95), 1e-6, 40 + side)
    n = side ** 3
    sz = (ol.C.c_uint * 3)(side, side, side)
    cr = np.zeros((24, n))
    co = np.zeros((24, n))
    REF.lib.ref_physical_constraints(ol.rows(cr), ol.rows(U), ol.C.c_uint(0), ol.P(pmin), ol.P(pmax), sz,
                                     ol.C.c_uint(bflag), ol.P(np.zeros(138 * n)))
    O.lib.orc_physical_constraints(ol.rows(co), ol.rows(U), ol.C.c_uint(0), ol.P(pmin), ol.P(pmax), sz,
                                   ol.C.c_uint(bflag), ol.P(np.zeros(288 * n)))
    a = mg.interior(cr, side)[:4]
    b = mg.interior(co, side)[:4]
    err = np.abs(a - b).max(axis=1) / np.abs(a).max(axis=1)
    assert err.max() <= 1e-12, err


@pytest.mark.parametrize("side,bflag", [(13, 0), (19, 63), (31, 21)])
def test_psi4_vs_reference_live(O, REF, side, bflag):
    """The restated Weyl scalar psi4 against the reference's own
    physconeqs.cpp (cons[4], cons[5] of physical_constraints)."""
    import sys
    sys.path.insert(0, os.path.join(HERE, "golden"))
    import make_golden as mg
    U, pmin, pmax = mg.golden_input(side, 2.0 / (side - 7), (0.1, -1.1, -0.95), 1e-6, 40 + side)
    n = side ** 3
    sz = (ol.C.c_uint * 3)(side, side, side)
    cr = np.zeros((24, n))
    REF.lib.ref_physical_constraints(ol.rows(cr), ol.rows(U), ol.C.c_uint(0), ol.P(pmin), ol.P(pmax), sz,
                                     ol.C.c_uint(bflag), ol.P(np.zeros(138 * n)))
    re, im = np.zeros(n), np.zeros(n)
    O.lib.orc_psi4(ol.P(re), ol.P(im), ol.rows(U), ol.C.c_uint(0), ol.P(pmin), ol.P(pmax), sz,
                   ol.C.c_uint(bflag), ol.P(np.zeros(288 * n)))
    a = mg.interior(cr, side)[4:6]
    b = mg.interior(np.concatenate([np.stack([re, im]), np.zeros((22, n))]), side)[:2]
    err = np.abs(a - b).max(axis=1) / np.abs(a).max(axis=1)
    assert err.max() <= 1e-12, err


def test_oracle_rk4_matches_reference_history_10_steps(O, REF):
    """The restated RHS inside the restated RK4 reproduces, after 10 steps,
    the constraint norms of the reference-RHS evolution in the committed
    history (to 1e-10 relative)."""
    import json
    import bssn_b200 as B  # mesh generator only (host code)
    with open(os.path.join(HERE, "golden", "constraint_history.json")) as f:
        gold = json.load(f)
    spec = B.generate_mesh(0, (8, 8, 8))
    mo = ol.MeshOracle(spec, O)
    Z = mo.initial_data()
    for _ in range(10):
        assert mo.rk4_step(Z, 0.25 * spec.h, ol.params()) == 0
    c = ol.oracle_constraints(spec, mo.unzip(Z), O)
    got = ol.l2_norms(spec, c, radii=(0.5, 0.5))
    ref = np.array([float.fromhex(x) for x in gold["history"][1]["norms"]])
    assert gold["history"][1]["step"] == 10
    assert np.abs(got - ref).max() / np.abs(ref).min() <= 1e-10, (got, ref)


def test_lowmem_rk4_step_bit_identical():
    """The block-by-block RK4 step (no unzipped arrays; used for the
    largest goldens) equals the oracle's RK4 step bit for bit, with the
    oracle's and with the reference's compiled right-hand side."""
    spec = ol.OracleMeshSpec(1, (2, 1, 1), seed=1, xmin=-8.25)
    mo = ol.MeshOracle(spec, ol.oracle())
    Z0 = mo.initial_data(eps=1e-8)
    ref = ol.reference()
    fns = [None] + ([ref.lib.ref_bssnRHS_blocks] if ref is not None else [])
    for fn in fns:
        A, Bz = Z0.copy(), Z0.copy()
        ws = mo.rk4_workspace()
        bufs = [np.zeros_like(Z0) for _ in range(3)]
        for _ in range(2):
            assert mo.rk4_step_ws(A, 0.25 * spec.h, ol.params(), ws, rhs_fn=fn) == 0
            assert mo.rk4_step_lowmem(Bz, 0.25 * spec.h, ol.params(), bufs, rhs_fn=fn) == 0
        assert np.array_equal(A.view(np.uint64), Bz.view(np.uint64))


def test_lowmem_constraint_norms_match():
    """Block-by-block constraint norms equal the unzipped computation to
    rounding of the summation order."""
    spec = ol.OracleMeshSpec(1, (2, 1, 1), seed=1, xmin=-8.25)
    O = ol.oracle()
    mo = ol.MeshOracle(spec, O)
    Z = mo.initial_data(eps=1e-6)
    ref = ol.l2_norms(spec, ol.oracle_constraints(spec, mo.unzip(Z), O))
    got = ol.constraint_norms_lowmem(spec, Z, O)
    assert np.allclose(got, ref, rtol=1e-13, atol=0), (got, ref)


def test_element_features_consistent_with_block_features():
    """The per-element features partition the block features' sublattice: a
    block's maxima are the largest of its elements' maxima, its smallest chi
    the smallest of theirs, and a one-element block (13^3) has the same 16
    features as its element (oracle against itself, on a mixed mesh with
    every side and a perturbed state)."""
    import ctypes as C
    spec = ol.OracleMeshSpec(1, (2, 1, 1), seed=1, xmin=-8.25)
    mo = ol.MeshOracle(spec, ol.oracle())
    rng = np.random.default_rng(3)
    Z = mo.initial_data(eps=1e-8, bh=(0.6, -4.1, -4.2, -0.6, -4.1, -4.2))
    Z += rng.standard_normal(Z.shape) * 1e-6
    U = mo.unzip(Z)
    sides = np.array([spec.blocks[b].sz for b in range(spec.nblocks)])
    assert set(sides.tolist()) == {13, 19, 31, 55}
    first = np.cumsum([0] + [((int(s) - 7) // 6) ** 3 for s in sides])
    fb = np.zeros((spec.nblocks, 16), dtype=np.float32)
    fe = np.zeros((first[-1], 16), dtype=np.float32)
    lib = mo.lib
    lib.orc_block_features(ol.rows(U), spec.blocks, spec.nblocks, fb.ctypes.data_as(C.c_void_p))
    lib.orc_element_features(ol.rows(U), spec.blocks, spec.nblocks, fe.ctypes.data_as(C.c_void_p))
    maxima = [0, 1, 2, 3, 4, 5, 6, 7, 8, 9, 13, 14]
    for b in range(spec.nblocks):
        e = fe[first[b]:first[b + 1]]
        assert np.array_equal(fb[b, maxima], e[:, maxima].max(axis=0)), b
        assert fb[b, 12] == e[:, 12].min(), b
        assert np.all(e[:, [10, 11, 15]] == fb[b, [10, 11, 15]]), b
        if sides[b] == 13:
            assert np.array_equal(fb[b], e[0]), b
