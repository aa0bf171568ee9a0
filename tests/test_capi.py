"""CPU tests of the C ABI library: it loads without a GPU, exports every
symbol include/*.h declares, and its host-only parts (mesh generator, tile
table) behave; no device calls."""
import ctypes as C
import os
import re
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIB = os.path.join(ROOT, "dendro-gr_b200", "lib", "libbssn_b200.so")


def declared_symbols():
    names = set()
    inc = os.path.join(ROOT, "include")
    for fn in os.listdir(inc):
        if not fn.endswith(".h"):
            continue
        text = open(os.path.join(inc, fn)).read()
        for m in re.finditer(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b(bssn_\w+)\s*\(", text, re.M):
            names.add(m.group(1))
    return names


def test_library_exports_declared_symbols():
    assert os.path.exists(LIB), "build with make -C dendro-gr_b200"
    out = subprocess.run(["nm", "-D", "--defined-only", LIB], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    decl = declared_symbols()
    assert len(decl) >= 20
    missing = decl - exported
    assert not missing, missing


def test_library_loads_and_reports():
    lib = C.CDLL(LIB)
    lib.bssn_version.restype = C.c_char_p
    assert b"sm_100a" in lib.bssn_version()
    assert lib.bssn_tile_count() >= 2


def test_invalid_arguments_are_rejected():
    import bssn_b200 as B
    assert B.lib.bssn_deriv644_f64(99, None, None, 0.1, None, 0, None) != 0
    assert B.lib.bssn_rk4_stage_f64(7, None, None, None, 10, 0.1, 1, 1e-4, None, None) != 0
    assert B.lib.bssn_mesh_create(None, 0, None, None) != 0


def _octants_covered(spec):
    M = [(g - 1) // 6 for g in spec.G]
    occ = np.zeros(M, dtype=np.int32)
    for b in range(spec.nblocks):
        blk = spec.blocks[b]
        w = (blk.sz - 7) // 6
        o = [blk.g0[d] // 6 for d in range(3)]
        occ[o[0]:o[0] + w, o[1]:o[1] + w, o[2]:o[2] + w] += 1
    return occ


def test_uniform_mesh_config1():
    import bssn_b200 as B
    spec = B.generate_mesh(0, (8, 8, 8))
    assert spec.nblocks == 512 and set(spec.sides.tolist()) == {13}
    assert spec.G == (49, 49, 49)
    assert abs(spec.h - 1.0 / 3.0) < 1e-15
    assert (_octants_covered(spec) == 1).all()
    nbound = sum(1 for b in range(spec.nblocks) if spec.blocks[b].bflag)
    assert nbound == 512 - 6 ** 3  # 296 boundary blocks


@pytest.mark.parametrize("dims,seed", [((7, 5, 4), 20261203), ((10, 10, 7), 20261203), ((2, 2, 1), 3)])
def test_mixed_mesh_tiles_the_box(dims, seed):
    import bssn_b200 as B
    spec = B.generate_mesh(1, dims, seed=seed)
    assert (_octants_covered(spec) == 1).all()
    offs = np.array([spec.blocks[b].offset for b in range(spec.nblocks)])
    assert (offs % 2 == 0).all() and (np.diff(offs) > 0).all()
    for b in range(spec.nblocks):
        blk = spec.blocks[b]
        s = blk.sz
        for d in range(3):
            assert abs((blk.ptmax[d] - blk.ptmin[d]) / (s - 1) - spec.h) < 1e-12
            lo = blk.g0[d] == 0
            hi = blk.g0[d] + s - 7 == spec.G[d] - 1
            assert bool(blk.bflag & (1 << 2 * d)) == lo
            assert bool(blk.bflag & (1 << (2 * d + 1))) == hi


def test_mixed_mesh_size_fractions():
    import bssn_b200 as B
    spec = B.generate_mesh(1, (10, 10, 7), seed=20261203)
    assert 19000 < spec.nblocks < 21500
    frac = np.array([(spec.sides == s).mean() for s in (13, 19, 31, 55)])
    assert np.abs(frac - np.array([0.7, 0.2, 0.08, 0.02])).max() < 0.02, frac


def test_tile_shared_memory_indexing_in_bounds():
    """Host replay of every tile's shared-memory reads (all brick extents,
    face cases and threads): no read may leave its array."""
    lib = C.CDLL(LIB)
    lib.bssn_tile_selfcheck.restype = C.c_long
    for t in range(lib.bssn_tile_count()):
        assert lib.bssn_tile_selfcheck(t) == 0, t
