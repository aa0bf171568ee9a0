"""Multi-level meshes on the CPU: the library's generator and host-built
level maps (csrc/levels.cu) against the independent geometric oracle
(oracle_levels.py) -- every ghost-fill source, owner and sync entry, applied
to the same seeded state, bit-identical -- and the interpolation exact on
polynomials of degree <= 6."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "dendro-gr_b200"))

import oracle_lib as ol  # noqa: E402
from oracle_levels import LevelOracle, lagrange_half  # noqa: E402

B = pytest.importorskip("bssn_b200")
from bssn_b200 import levels as LV  # noqa: E402

MESHES = {
    "two": ((4, 4, 4), [((2, 2, 2), (4, 4, 4))]),
    "three": ((6, 6, 6), [((2, 4, 2), (6, 4, 8)), ((6, 10, 6), (4, 2, 6))]),
}


@pytest.fixture(scope="module")
def O():
    return ol.oracle()


def eval_maps(maps, Z, W):
    """The library's maps applied in numpy: ghost fill and sync."""
    itp = maps["interp"]

    def value(src):
        out = np.zeros((Z.shape[0], len(src)))
        pos = src >= 0
        out[:, pos] = Z[:, src[pos]]
        ent = itp[-2 - src[src <= -2]]
        sel = np.nonzero(src <= -2)[0]
        n = np.where(ent[:, 4:7] >= 0, 7, 1)
        for pat in np.unique(n @ np.array([1, 10, 100])):
            m = (n @ np.array([1, 10, 100])) == pat
            e, s = ent[m], sel[m]
            nx, ny, nz = pat % 10, (pat // 10) % 10, pat // 100
            w = [W[np.maximum(e[:, 4 + d], 0)] if (nx, ny, nz)[d] == 7 else np.ones((len(e), 1)) for d in range(3)]
            tz = None
            for c in range(nz):
                ty = None
                for b in range(ny):
                    tx = None
                    for a in range(nx):
                        t = w[0][:, a] * Z[:, e[:, 0] + a * e[:, 1] + b * e[:, 2] + c * e[:, 3]]
                        tx = t if a == 0 else tx + t
                    t = w[1][:, b] * tx
                    ty = t if b == 0 else ty + t
                t = w[2][:, c] * ty
                tz = t if c == 0 else tz + t
            out[:, s] = tz
        return out

    return value


@pytest.mark.parametrize("name", sorted(MESHES))
def test_generator_tiles_levels(name):
    M0, boxes = MESHES[name]
    spec = LV.generate_levels(M0, boxes)
    bl = spec.as_numpy()
    assert set(bl["sz"].tolist()) <= {13, 19, 31, 55}
    assert (bl["bflag"][bl["level"] > 0] == 0).all()
    assert spec.h == spec.h0 / 2 ** len(boxes)
    # the block offsets are increasing and non-overlapping
    ends = bl["offset"] + bl["sz"].astype(np.int64) ** 3
    assert (bl["offset"][1:] >= ends[:-1]).all()
    LO = LevelOracle(spec, ol.oracle())
    for l, (lo, n) in enumerate(LO.boxes):
        under = np.zeros(tuple(n[::-1]), dtype=bool)
        if l + 1 < LO.L:
            clo, cn = LO.boxes[l + 1][0] // 2 - lo, LO.boxes[l + 1][1] // 2
            under[clo[2]:clo[2] + cn[2], clo[1]:clo[1] + cn[1], clo[0]:clo[0] + cn[0]] = True
        assert ((LO.octs[l] >= 0) == ~under).all(), l
    assert LO.n_nodes == spec.n_nodes


@pytest.mark.parametrize("name", sorted(MESHES))
def test_maps_match_oracle(name, O):
    M0, boxes = MESHES[name]
    spec = LV.generate_levels(M0, boxes)
    LO = LevelOracle(spec, O)
    maps = LV.level_maps(spec)
    W = lagrange_half()
    rng = np.random.default_rng(7)
    Z = rng.standard_normal((3, spec.n_nodes))
    value = eval_maps(maps, Z, W)
    # ghost fill
    Z24 = np.zeros((ol.NVARS, spec.n_nodes))
    Z24[:3] = Z
    ref = LO.unzip(Z24)[:3]
    got = value(maps["unzip_src"])
    assert np.array_equal(got.view(np.uint64), ref.view(np.uint64))
    # owners
    assert np.array_equal(maps["zip_src"], LO.owners())
    # sync: injections then prolongations, in the library's list order
    S = Z.copy()
    inj, pro = maps["inject"], maps["prolong"]
    lv_node = np.searchsorted(np.array(LO.offsets[1:]), inj[:, 0], side="right")
    for l in sorted(set(lv_node.tolist()), reverse=True):
        m = lv_node == l
        S[:, inj[m, 0]] = S[:, inj[m, 1]]
    pl = np.searchsorted(np.array(LO.offsets[1:]), pro[:, 0], side="right")
    for l in sorted(set(pl.tolist())):
        m = pl == l
        S[:, pro[m, 0]] = eval_maps(maps, S, W)(pro[m, 1])
    Z24 = np.zeros((ol.NVARS, spec.n_nodes))
    Z24[:3] = Z
    ref = LO.sync(Z24)[:3]
    assert np.array_equal(S.view(np.uint64), ref.view(np.uint64))


def test_interpolation_exact_on_degree_6(O):
    """A degree-6 polynomial in x, y, z per level grid: the ghost fill of
    the finer blocks reproduces it outside their box (rounding only)."""
    M0, boxes = MESHES["two"]
    spec = LV.generate_levels(M0, boxes)
    LO = LevelOracle(spec, O)
    Z = np.zeros((ol.NVARS, spec.n_nodes))

    def poly(x, y, z):
        return 0.3 + x ** 6 / 4096 - 0.2 * x * y ** 3 * z ** 2 / 512 + 0.1 * y ** 5 / 1024 - z ** 4 / 256 + x * y

    coords = []
    for l, (lo, n) in enumerate(LO.boxes):
        h = spec.h0 / 2 ** l
        d = LO.dims[l]
        z, y, x = np.meshgrid(*[np.arange(k) for k in d[::-1]], indexing="ij")
        pts = [spec.xmin + (OCTL + o) * h for OCTL, o in zip((x.ravel(), y.ravel(), z.ravel()), 6 * lo)]
        coords.append(pts)
        Z[0, LO.offsets[l]:LO.offsets[l] + int(np.prod(d))] = poly(*pts)
    P = LO.unzip(Z)
    bl = spec.as_numpy()
    worst = 0.0
    for b in np.nonzero(bl["level"] == 1)[0]:
        s = int(bl["sz"][b])
        h = spec.h0 / 2
        i = np.arange(s)
        zz, yy, xx = np.meshgrid(i, i, i, indexing="ij")
        q = np.stack([xx.ravel(), yy.ravel(), zz.ravel()], axis=1) + bl["g0"][b] - 3
        x, y, z = [spec.xmin + q[:, k] * h for k in range(3)]
        exact = poly(x, y, z)
        got = P[0, int(bl["offset"][b]):int(bl["offset"][b]) + s ** 3]
        worst = max(worst, np.abs(got - exact).max() / np.abs(exact).max())
    assert worst < 1e-12, worst


def test_regrid_policy():
    """Box hierarchies from refine flags: nothing flagged -> one level;
    flagged finest blocks keep their level and add one finer; a flag near
    the domain boundary is covered up to the nesting clamp; every result is
    a valid hierarchy (the generator accepts it)."""
    M0, boxes = MESHES["two"]
    spec = LV.generate_levels(M0, boxes)
    bl = spec.as_numpy()
    assert LV.regrid_boxes(spec, np.zeros(spec.nblocks)) == []
    fine = (bl["level"] == 1).astype(np.uint8)
    nb = LV.regrid_boxes(spec, fine)
    assert nb[0] == ((2, 2, 2), (4, 4, 4)) and nb[1] == ((6, 6, 6), (4, 4, 4))
    assert LV.regrid_boxes(spec, fine, max_levels=2) == [((2, 2, 2), (4, 4, 4))]
    corner = np.zeros(spec.nblocks, dtype=np.uint8)
    corner[np.nonzero((bl["level"] == 0) & np.all(bl["g0"] == 0, axis=1))[0]] = 1
    nb = LV.regrid_boxes(spec, corner)
    assert nb == [((2, 2, 2), (2, 2, 2))]
    for flags in (fine, corner, np.ones(spec.nblocks)):
        LV.generate_levels(M0, LV.regrid_boxes(spec, flags))
    # coarsening hysteresis: kept finest blocks hold their level (the box
    # stays) without adding a finer one; kept flags on level 0 change nothing
    none = np.zeros(spec.nblocks, dtype=np.uint8)
    assert LV.regrid_boxes(spec, none, keep=fine) == [((2, 2, 2), (4, 4, 4))]
    assert LV.regrid_boxes(spec, none, keep=(bl["level"] == 0)) == []
    assert LV.regrid_boxes(spec, fine, keep=fine) == LV.regrid_boxes(spec, fine)


PATCHES = ((8, 4, 4), [(1, 0, (2, 2, 2), (4, 4, 4)), (1, 0, (10, 2, 2), (4, 4, 4)),
                       (2, 1, (6, 6, 6), (4, 4, 4))])


def test_patch_maps_match_oracle(O):
    """Two separate level-1 patches (one with a level-2 child): the
    library's maps against the patch-aware oracle, bit for bit."""
    spec = LV.generate_patches(*PATCHES)
    LO = LevelOracle(spec, O)
    maps = LV.level_maps(spec)
    W = lagrange_half()
    rng = np.random.default_rng(9)
    Z = rng.standard_normal((3, spec.n_nodes))
    Z24 = np.zeros((ol.NVARS, spec.n_nodes))
    Z24[:3] = Z
    value = eval_maps(maps, Z, W)
    ref = LO.unzip(Z24)[:3]
    assert np.array_equal(value(maps["unzip_src"]).view(np.uint64), ref.view(np.uint64))
    assert np.array_equal(maps["zip_src"], LO.owners())
    # sync through the maps: restriction by source level (finest first),
    # then prolongation by level (coarsest first)
    patch_of = lambda nodes: np.searchsorted(np.array(LO.offsets[1:]), nodes, side="right")  # noqa: E731
    lev = np.array(LO.level)
    S = Z.copy()
    inj, pro = maps["inject"], maps["prolong"]
    il = lev[patch_of(inj[:, 1])]
    for l in sorted(set(il.tolist()), reverse=True):
        m = il == l
        S[:, inj[m, 0]] = S[:, inj[m, 1]]
    pl = lev[patch_of(pro[:, 0])]
    for l in sorted(set(pl.tolist())):
        m = pl == l
        S[:, pro[m, 0]] = eval_maps(maps, S, W)(pro[m, 1])
    ref = LO.sync(Z24.copy())[:3]
    assert np.array_equal(S.view(np.uint64), ref.view(np.uint64))


def test_patch_rules():
    """Invalid hierarchies are refused: patches of one level too close,
    a child without margin, a parent of the wrong level."""
    M0 = (8, 4, 4)
    with pytest.raises(B.BssnError):  # level-1 patches touching (less than a parent octant apart)
        LV.generate_patches(M0, [(1, 0, (2, 2, 2), (4, 4, 4)), (1, 0, (6, 2, 2), (4, 4, 4))])
    LV.generate_patches(M0, [(1, 0, (2, 2, 2), (4, 4, 4)), (1, 0, (8, 2, 2), (4, 4, 4))])  # one apart: valid
    with pytest.raises(B.BssnError):  # no margin inside the parent
        LV.generate_patches(M0, [(1, 0, (0, 2, 2), (4, 4, 4))])
    with pytest.raises(B.BssnError):  # parent of the wrong level
        LV.generate_patches(M0, [(1, 0, (2, 2, 2), (4, 4, 4)), (1, 1, (6, 6, 6), (4, 4, 4))])


def test_regrid_patches_clusters():
    """Refinement in two separate places gives two patches per level (each
    refined again where its fine blocks are flagged); nothing flagged gives
    none; every result is a valid hierarchy."""
    M0 = (12, 4, 4)
    spec = LV.generate_patches(M0, [(1, 0, (2, 2, 2), (4, 4, 4)), (1, 0, (16, 2, 2), (4, 4, 4))])
    bl = spec.as_numpy()
    assert LV.regrid_patches(spec, np.zeros(spec.nblocks)) == []
    pt = LV.regrid_patches(spec, (bl["level"] == 1).astype(np.uint8))
    lev = [p[0] for p in pt]
    assert lev.count(1) == 2 and lev.count(2) == 2
    for k, par, lo, n in pt:  # children nest in their own parent
        if k == 2:
            plo, pn = np.array(pt[par - 1][2]), np.array(pt[par - 1][3])
            assert np.all(np.array(lo) // 2 >= plo + 1) and np.all((np.array(lo) + n) // 2 <= plo + pn - 1)
    LV.generate_patches(M0, pt)
    # flags only on the level-0 blocks at the two ends: two level-1 patches
    ends = np.zeros(spec.nblocks, dtype=np.uint8)
    for b in np.nonzero(bl["level"] == 0)[0]:
        o, w = bl["g0"][b] // 6, (int(bl["sz"][b]) - 7) // 6
        if o[0] <= 1 < o[0] + w or o[0] <= 10 < o[0] + w:
            ends[b] = 1
    pt = LV.regrid_patches(spec, ends, max_levels=2)
    assert [p[0] for p in pt] == [1, 1]
    LV.generate_patches(M0, pt)


def test_evolve_norm_mask_counts_each_point_once():
    """The full-evolution driver's constraint-norm mask: with no puncture
    radii it holds every independent point of a level mesh exactly once (the
    zone-owned nodes; patch-boundary nodes are filled from the coarser level
    and counted there where they coincide with a coarse node), and its boxes
    are the nested centred boxes."""
    torch = pytest.importorskip("torch")
    from bssn_b200 import evolve as EV
    from bssn_b200 import levels as LV
    assert EV.nested_boxes(24, 3) == [((12,) * 3, (24,) * 3), ((36,) * 3, (24,) * 3)]
    spec = LV.generate_levels((4, 4, 4), EV.nested_boxes(4, 3), xmin=-8.0, L=16.0)
    m = EV.norm_mask(spec, radii=(0.0, 0.0))
    pts = set()
    for g in spec.grids():
        nx, ny, nz = g["dims"]
        for k in range(nz):
            for j in range(ny):
                for i in range(nx):
                    if g["level"] > 0 and (min(i, j, k) == 0 or i == nx - 1 or j == ny - 1 or k == nz - 1):
                        continue
                    pts.add(tuple(round((g["origin"][d] + e * g["h"]) * 1024) for d, e in enumerate((i, j, k))))
    assert int(m.sum()) == len(pts)
    m2 = EV.norm_mask(spec)
    assert 0 < int(m2.sum()) < int(m.sum())


def test_evolve_remesh_rule():
    """The driver rebuilds the mesh only when the regrid asks for a level
    more or less, a box reaching outside the current one, or a current box
    more than twice the volume asked for."""
    from bssn_b200 import evolve as EV
    cur = [((2, 2, 2), (8, 8, 8)), ((6, 6, 6), (8, 8, 8))]
    assert not EV.needs_remesh(cur, cur)
    assert not EV.needs_remesh(cur, [((2, 2, 2), (8, 8, 6)), ((6, 6, 6), (8, 8, 8))])
    assert EV.needs_remesh(cur, cur[:1])
    assert EV.needs_remesh(cur, [((0, 2, 2), (8, 8, 8)), ((6, 6, 6), (8, 8, 8))])
    assert EV.needs_remesh(cur, [((2, 2, 2), (8, 8, 10)), ((6, 6, 6), (8, 8, 8))])
    assert EV.needs_remesh(cur, [((2, 2, 2), (4, 8, 6)), ((6, 6, 6), (8, 8, 8))])


def test_remesh_decision_thresholds():
    """The learned decision's thresholds (host logic): at most half the
    missed-refinement budget of the validation positives lies at or below lo,
    at most the false-refinement budget of the negatives at or above hi, and
    lo <= hi."""
    from bssn_b200.remesh_train import pick_thresholds
    rng = np.random.default_rng(4)
    y = (rng.random(40000) < 0.3).astype(np.float32)
    p = np.clip(np.where(y > 0.5, rng.beta(8, 2, y.size), rng.beta(2, 8, y.size)), 0, 1).astype(np.float32)
    for fn, fp in ((1e-3, 1e-3), (2e-4, 1e-2)):
        lo, hi = pick_thresholds(p, y, fn_target=fn, fp_target=fp)
        pos, neg = p[y > 0.5], p[y < 0.5]
        assert lo <= hi
        assert (pos <= lo).mean() <= fn / 2
        assert (neg >= hi).mean() <= fp
