"""Multi-level meshes (csrc/levels.cu; the level rules are documented beside
BssnLevelBox in include/bssn_b200.h): nested level boxes with 2:1
refinement, blocks tiling each level's region, the zipped state the
concatenation of one dense node grid per level.

    spec = generate_levels(M0=(4, 4, 4), boxes=[((2, 2, 2), (4, 4, 4))])
    mesh = Mesh(spec)                        # level maps uploaded
    U = torch.zeros((24, spec.n_nodes), dtype=torch.float64, device="cuda")
    initial_data_levels(U, spec)             # per level grid, then level sync
    plan = RK4Plan(mesh, default_params()); plan.step(U, 0.25 * spec.h)
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field

import numpy as np

from . import NVARS, BssnBlockDesc, MeshSpec, check, lib, stream_ptr

OCT = 6


class BssnLevelBox(C.Structure):
    _fields_ = [("lo", C.c_int32 * 3), ("n", C.c_int32 * 3)]


class BssnPatch(C.Structure):
    _fields_ = [("level", C.c_int32), ("parent", C.c_int32), ("lo", C.c_int32 * 3), ("n", C.c_int32 * 3)]


lib.bssn_mesh_generate_levels.argtypes = [C.c_int, C.POINTER(C.c_int32), C.POINTER(BssnLevelBox), C.c_double,
                                          C.c_double, C.POINTER(BssnBlockDesc), C.POINTER(C.c_int),
                                          C.POINTER(C.c_int64)]
lib.bssn_mesh_create_levels.argtypes = [C.POINTER(BssnBlockDesc), C.c_int, C.c_int, C.POINTER(C.c_int32),
                                        C.POINTER(BssnLevelBox), C.POINTER(C.c_void_p)]
lib.bssn_mesh_levels_sync.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
lib.bssn_levels_maps.argtypes = [C.POINTER(BssnBlockDesc), C.c_int, C.c_int, C.POINTER(C.c_int32),
                                 C.POINTER(BssnLevelBox), C.POINTER(C.c_int64)] + [C.c_void_p] * 5
lib.bssn_mesh_generate_patches.argtypes = [C.c_int, C.POINTER(C.c_int32), C.POINTER(BssnPatch), C.c_double,
                                           C.c_double, C.POINTER(BssnBlockDesc), C.POINTER(C.c_int),
                                           C.POINTER(C.c_int64)]
lib.bssn_mesh_generate_patches_w.argtypes = [C.c_int, C.POINTER(C.c_int32), C.POINTER(BssnPatch), C.c_double,
                                             C.c_double, C.c_int, C.POINTER(BssnBlockDesc), C.POINTER(C.c_int),
                                             C.POINTER(C.c_int64)]
lib.bssn_mesh_create_patches.argtypes = [C.POINTER(BssnBlockDesc), C.c_int, C.c_int, C.POINTER(C.c_int32),
                                         C.POINTER(BssnPatch), C.POINTER(C.c_void_p)]
lib.bssn_patches_maps.argtypes = [C.POINTER(BssnBlockDesc), C.c_int, C.c_int, C.POINTER(C.c_int32),
                                  C.POINTER(BssnPatch), C.POINTER(C.c_int64)] + [C.c_void_p] * 5


@dataclass
class LevelMeshSpec(MeshSpec):
    """A MeshSpec whose zipped state spans several level grids.  `h` is the
    finest spacing (the time step's), `h0` level 0's; G = (n_nodes, 1, 1)."""
    M0: tuple = (1, 1, 1)
    boxes: list = field(default_factory=list)   # [(lo, n)] per level, level octants
    h0: float = 0.0
    # [(level, parent, lo, n)] per patch when a level holds several patches
    # (None: one patch per level, the boxes above)
    patches: list = None
    # largest block, in octants per axis (8: sides up to 55)
    max_w: int = 8

    @property
    def patch_list(self):
        if self.patches is not None:
            return list(self.patches)
        return [(l, l - 1, lo, n) for l, (lo, n) in enumerate(self.boxes)]

    @property
    def nlevels(self):
        return 1 + max(p[0] for p in self.patch_list)

    def c_patches(self):
        pl = self.patch_list
        arr = (BssnPatch * len(pl))()
        for i, (lev, par, lo, n) in enumerate(pl):
            arr[i].level, arr[i].parent = lev, par
            arr[i].lo[:] = list(lo)
            arr[i].n[:] = list(n)
        return arr

    def c_boxes(self):
        arr = (BssnLevelBox * len(self.boxes))()
        for l, (lo, n) in enumerate(self.boxes):
            arr[l].lo[:] = list(lo)
            arr[l].n[:] = list(n)
        return arr

    def grids(self):
        """Per patch: dict(level, lo, n, dims, offset, h, origin) of its node grid."""
        out, off = [], 0
        for lev, _, lo, n in self.patch_list:
            dims = tuple(OCT * int(x) + 1 for x in n)
            h = self.h0 / 2 ** lev
            origin = tuple(self.xmin + OCT * int(lo[d]) * h for d in range(3))
            out.append(dict(level=lev, lo=tuple(lo), n=tuple(n), dims=dims, offset=off, h=h, origin=origin))
            off += dims[0] * dims[1] * dims[2]
        return out


def generate_levels(M0, boxes, xmin=-8.0, L=16.0, max_w=8):
    """Level 0 = the domain [xmin, xmin + L]^3 in M0 octants per axis; boxes
    = [(lo, n)] of levels 1.. in their own octants; blocks of at most max_w
    octants per axis."""
    allb = [((0, 0, 0), tuple(M0))] + [(tuple(lo), tuple(n)) for lo, n in boxes]
    h0 = L / (OCT * M0[0])
    spec = LevelMeshSpec(None, 0, (0, 1, 1), h0 / 2 ** (len(allb) - 1), xmin, None, None,
                         tuple(M0), allb, h0, None, int(max_w))
    cp = spec.c_patches()
    M = (C.c_int32 * 3)(*M0)
    n = C.c_int(0)
    nn = C.c_int64(0)
    check(lib.bssn_mesh_generate_patches_w(len(allb), M, cp, xmin, h0, int(max_w), None, C.byref(n), C.byref(nn)),
          "mesh_generate_levels")
    blocks = (BssnBlockDesc * n.value)()
    check(lib.bssn_mesh_generate_patches_w(len(allb), M, cp, xmin, h0, int(max_w), blocks, C.byref(n),
                                           C.byref(nn)), "mesh_generate_levels")
    spec.blocks, spec.nblocks = blocks, n.value
    spec.G = (int(nn.value), 1, 1)
    spec.sides = np.array([blocks[b].sz for b in range(n.value)], dtype=np.int32)
    return spec


def generate_patches(M0, patches, xmin=-8.0, L=16.0, max_w=8):
    """Patch 0 = the domain [xmin, xmin + L]^3 in M0 octants per axis;
    patches = [(level, parent, lo, n)] of patches 1.. (parents listed first,
    boxes in their own level's octants); blocks of at most max_w octants per
    axis."""
    allp = [(0, -1, (0, 0, 0), tuple(M0))] + [(int(a), int(b), tuple(lo), tuple(n)) for a, b, lo, n in patches]
    h0 = L / (OCT * M0[0])
    nlev = 1 + max(p[0] for p in allp)
    spec = LevelMeshSpec(None, 0, (0, 1, 1), h0 / 2 ** (nlev - 1), xmin, None, None, tuple(M0), [], h0, allp,
                         int(max_w))
    cp = spec.c_patches()
    M = (C.c_int32 * 3)(*M0)
    n = C.c_int(0)
    nn = C.c_int64(0)
    check(lib.bssn_mesh_generate_patches_w(len(allp), M, cp, xmin, h0, int(max_w), None, C.byref(n), C.byref(nn)),
          "mesh_generate_patches")
    blocks = (BssnBlockDesc * n.value)()
    check(lib.bssn_mesh_generate_patches_w(len(allp), M, cp, xmin, h0, int(max_w), blocks, C.byref(n),
                                           C.byref(nn)), "mesh_generate_patches")
    spec.blocks, spec.nblocks = blocks, n.value
    spec.G = (int(nn.value), 1, 1)
    spec.sides = np.array([blocks[b].sz for b in range(n.value)], dtype=np.int32)
    return spec


def create_mesh_handle(spec: LevelMeshSpec):
    h = C.c_void_p()
    M = (C.c_int32 * 3)(*spec.M0)
    pl = spec.patch_list
    check(lib.bssn_mesh_create_patches(spec.blocks, spec.nblocks, len(pl), M, spec.c_patches(), C.byref(h)),
          "mesh_create_patches")
    return h


def _rows(U, off=0):
    n = U.shape[1]
    return (C.c_void_p * NVARS)(*[U.data_ptr() + (v * n + off) * 8 for v in range(NVARS)])


def sync(mesh, U, stream=None):
    """Level sync of the zipped state U ((24, n_nodes) CUDA tensor)."""
    check(lib.bssn_mesh_levels_sync(mesh.h, _rows(U), NVARS, stream_ptr(stream)), "mesh_levels_sync")


def initial_data_levels(U, spec: LevelMeshSpec, mesh=None, bh=(1.0, 0.0, 0.0, -1.0, 0.0, 0.0), m1=0.5,
                        m2=0.5, chi_floor=1e-4, eps=1e-8, seed=20261203, stream=None):
    """Brill-Lindquist data on every patch grid (noise seed + patch index),
    then the level sync when a mesh handle is given."""
    b = (C.c_double * 6)(*bh)
    for l, g in enumerate(spec.grids()):
        G = (C.c_int32 * 3)(*g["dims"])
        xm = (C.c_double * 3)(*g["origin"])
        check(lib.bssn_initial_data_f64(_rows(U, g["offset"]), G, xm, g["h"], b, m1, m2, chi_floor, eps,
                                        seed + l, stream_ptr(stream)), "initial_data")
    if mesh is not None:
        sync(mesh, U, stream)


def level_maps(spec: LevelMeshSpec):
    """The library's host-built maps as numpy arrays (for tests)."""
    M = (C.c_int32 * 3)(*spec.M0)
    cb = spec.c_patches()
    npch = len(spec.patch_list)
    sizes = (C.c_int64 * 5)()
    check(lib.bssn_patches_maps(spec.blocks, spec.nblocks, npch, M, cb, sizes, None, None, None, None,
                                None), "patches_maps")
    npad, nn, ninj, npro, nint = [int(x) for x in sizes]
    unz = np.zeros(npad, dtype=np.int64)
    zp = np.zeros(nn, dtype=np.int64)
    inj = np.zeros((max(ninj, 1), 2), dtype=np.int64)
    pro = np.zeros((max(npro, 1), 2), dtype=np.int64)
    itp = np.zeros((max(nint, 1), 7), dtype=np.int64)
    check(lib.bssn_patches_maps(spec.blocks, spec.nblocks, npch, M, cb, sizes, unz.ctypes.data,
                                zp.ctypes.data, inj.ctypes.data, pro.ctypes.data, itp.ctypes.data), "patches_maps")
    return dict(unzip_src=unz, zip_src=zp, inject=inj[:ninj], prolong=pro[:npro], interp=itp[:nint])


lib.bssn_levels_transfer.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]


def transfer(mesh_from, U_old, mesh_to, U_new, stream=None):
    """U_new on mesh_to's hierarchy from U_old on mesh_from's (same level-0
    domain): same-level copies where the old grid has the node, else the
    coarse node or interpolation from the new coarser level; then the level
    sync.  Blocking."""
    check(lib.bssn_levels_transfer(mesh_from.h, _rows(U_old), mesh_to.h, _rows(U_new), NVARS,
                                   stream_ptr(stream)), "levels_transfer")


def regrid_boxes(spec: LevelMeshSpec, flags, max_levels=None, keep=None, max_n=None):
    """New level boxes (levels 1.., level-l octants) from per-block refine
    flags, the box-hierarchy form of the reference's remesh (refine where
    the test flags a block, coarsen where nothing asks for the level):

    * level l+1 must cover every flagged level-l block, every flagged level-
      (l+1) block (still wanted fine), and level l+2's new box with one
      level-(l+1) octant of margin;
    * each box is widened by one parent octant (two of its own) on every
      side, aligned to parent octant corners, and clamped inside its parent
      with one parent octant of margin (flags closer to the domain boundary than that are
      covered only as far as the clamp allows);
    * a level nothing asks for is dropped with every finer one; at most one
      level finer than the current finest is added (max_levels caps the
      total);
    * keep (optional): blocks that hold their level without refining (the
      reference's coarsening hysteresis: a block coarsens only when its
      wavelet score is below BSSN_DENDRO_AMR_FAC * tol, BSSN_GR/src/
      dataUtils.cpp:413-480); level l must cover its kept blocks too;
    * max_n (optional, even): at most max_n own octants per axis and level,
      the box shrunk about its centre (the size cap that the reference's
      maximum depth gives an octree).
    Returns [(lo, n)] for levels 1.. (empty: a single-level mesh)."""
    flags = np.asarray(flags).astype(bool)
    held = flags if keep is None else flags | np.asarray(keep).astype(bool)
    bl = spec.as_numpy()
    L = spec.nlevels
    top = L + 1 if max_levels is None else min(L + 1, max_levels)
    req = [None] * (top + 1)   # req[l]: (lo, hi) of level l in level-l octants, hi exclusive
    for l in range(top - 1, 0, -1):
        parts = []
        for lev, scale, fl in ((l - 1, 2, flags), (l, 1, held)):
            for b in np.nonzero(fl & (bl["level"] == lev))[0]:
                o = np.asarray(bl["g0"][b], dtype=np.int64) // OCT
                w = (int(bl["sz"][b]) - 7) // OCT
                parts.append((o * scale, (o + w) * scale))
        if req[l + 1] is not None:
            lo, hi = req[l + 1]
            parts.append((lo // 2 - 1, -(-hi // 2) + 1))
        if not parts:
            continue
        lo = np.min([p[0] for p in parts], axis=0) - 2
        hi = np.max([p[1] for p in parts], axis=0) + 2
        req[l] = (lo - (lo % 2), hi + (hi % 2))
    boxes = []
    plo, pn = np.zeros(3, dtype=np.int64), np.asarray(spec.M0, dtype=np.int64)
    for l in range(1, top):
        if req[l] is None:
            break
        lo, hi = req[l]
        lo = np.maximum(lo, 2 * (plo + 1))
        hi = np.minimum(hi, 2 * (plo + pn - 1))
        if max_n is not None:
            over = hi - lo > max_n
            c = ((lo + hi) // 4) * 2
            lo = np.where(over, np.maximum(c - max_n // 2, 2 * (plo + 1)), lo)
            hi = np.where(over, np.minimum(lo + max_n, 2 * (plo + pn - 1)), hi)
        if np.any(hi - lo < 2):
            break
        boxes.append((tuple(int(x) for x in lo), tuple(int(x) for x in hi - lo)))
        plo, pn = lo, hi - lo
    return boxes


def remesh(mesh, U, flags, max_levels=None, patches=False, stream=None, keep=None, max_n=None):
    """Regrid a level mesh from refine flags and carry the state over:
    returns (spec, mesh, U) on the new hierarchy (the old mesh and state are
    left as they are).  patches: one patch per cluster of refinement
    (regrid_patches) instead of one box per level (regrid_boxes, which also
    takes the blocks that keep their level)."""
    import torch
    spec = mesh.spec
    f = flags.cpu().numpy() if hasattr(flags, "cpu") else flags
    from . import Mesh
    L = spec.h0 * OCT * spec.M0[0]
    if patches:
        new = generate_patches(spec.M0, regrid_patches(spec, f, max_levels), xmin=spec.xmin, L=L, max_w=spec.max_w)
    else:
        new = generate_levels(spec.M0, regrid_boxes(spec, f, max_levels, keep=keep, max_n=max_n), xmin=spec.xmin, L=L,
                              max_w=spec.max_w)
    nmesh = Mesh(new)
    V = torch.empty((NVARS, new.n_nodes), dtype=torch.float64, device=U.device)
    transfer(mesh, U, nmesh, V, stream)
    return new, nmesh, V


def regrid_patches(spec: LevelMeshSpec, flags, max_levels=None):
    """Patches (level, parent, lo, n) from per-block refine flags, one patch
    per connected cluster of refinement, the multi-region form of
    regrid_boxes (octree-like: separate sources get separate patches):

    * level k needs the level-(k-1) octants of every flagged level-(k-1)
      block, of every flagged level-k block (kept fine), and of every new
      level-(k+1) patch (widened by one level-k octant, so it nests);
    * flagged octants are widened by one parent octant, and all of them are
      grouped into 26-connected clusters; each cluster's bounding box is a
      patch, clamped to the region where level-k patches nest inside the
      domain; patches closer than one parent octant are merged;
    * levels are built finest first, so every patch lies inside the patch of
      the level below that holds it; at most one level finer than the
      current finest is added (max_levels caps the total).
    Returns the patches after patch 0 (parents listed first)."""
    flags = np.asarray(flags).astype(bool)
    bl = spec.as_numpy()
    L = spec.nlevels
    top = L + 1 if max_levels is None else min(L + 1, max_levels)
    M0 = np.asarray(spec.M0, dtype=np.int64)
    # allowed [A, B) for level-k patch boxes, in level-(k-1) octants
    A, Bnd = {1: np.ones(3, dtype=np.int64)}, {1: M0 - 1}
    for k in range(2, top):
        A[k], Bnd[k] = 2 * A[k - 1] + 1, 2 * Bnd[k - 1] - 1
    per_level = {}          # level -> list of (lo, hi) in level-k octants
    for k in range(top - 1, 0, -1):
        cells = set()
        for lev, scale in ((k - 1, 1), (k, 0)):
            for b in np.nonzero(flags & (bl["level"] == lev))[0]:
                o = np.asarray(bl["g0"][b], dtype=np.int64) // OCT
                w = (int(bl["sz"][b]) - 7) // OCT
                if scale == 0:  # level-k block -> its level-(k-1) octants
                    lo, hi = o // 2, -(-(o + w) // 2)
                else:
                    lo, hi = o, o + w
                lo, hi = lo - 1, hi + 1  # widened by one parent octant
                for x in range(lo[0], hi[0]):
                    for y in range(lo[1], hi[1]):
                        for z in range(lo[2], hi[2]):
                            cells.add((x, y, z))
        for lo, hi in per_level.get(k + 1, []):  # finer patches, in level-(k-1) octants, widened
            clo, chi = lo // 4 - 1, -(-hi // 4) + 1
            for x in range(clo[0], chi[0]):
                for y in range(clo[1], chi[1]):
                    for z in range(clo[2], chi[2]):
                        cells.add((x, y, z))
        if not cells:
            continue
        # 26-connected clusters
        boxes, seen = [], set()
        for c in cells:
            if c in seen:
                continue
            comp, stack = [], [c]
            seen.add(c)
            while stack:
                u = stack.pop()
                comp.append(u)
                for dx in (-1, 0, 1):
                    for dy in (-1, 0, 1):
                        for dz in (-1, 0, 1):
                            v = (u[0] + dx, u[1] + dy, u[2] + dz)
                            if v in cells and v not in seen:
                                seen.add(v)
                                stack.append(v)
            a = np.array(comp, dtype=np.int64)
            lo = np.maximum(a.min(axis=0), A[k])
            hi = np.minimum(a.max(axis=0) + 1, Bnd[k])
            if np.all(hi > lo):
                boxes.append([lo, hi])
        # merge boxes closer than one parent octant (in level-(k-1) octants)
        merged = True
        while merged:
            merged = False
            for i in range(len(boxes)):
                for j in range(i + 1, len(boxes)):
                    (alo, ahi), (blo, bhi) = boxes[i], boxes[j]
                    if np.all((alo < bhi + 1) & (blo < ahi + 1)):
                        boxes[i] = [np.minimum(alo, blo), np.maximum(ahi, bhi)]
                        del boxes[j]
                        merged = True
                        break
                if merged:
                    break
        per_level[k] = [(2 * lo, 2 * hi) for lo, hi in boxes]  # level-k octants
    out = []
    index = {0: [(0, np.zeros(3, dtype=np.int64), 2 * M0)]}  # level -> [(patch, lo, hi) in next-level units]
    for k in range(1, top):
        if k not in per_level or not index.get(k - 1):
            break
        index[k] = []
        for lo, hi in per_level[k]:
            parent = None
            for pi, plo, phi in index[k - 1]:
                if np.all(lo >= plo) and np.all(hi <= phi):
                    parent = pi
                    break
            if parent is None:
                continue  # cannot nest (clamped away): dropped with its subtree
            pid = len(out) + 1
            out.append((k, parent, tuple(int(v) for v in lo), tuple(int(v) for v in hi - lo)))
            index[k].append((pid, 2 * lo, 2 * hi))
    return out
