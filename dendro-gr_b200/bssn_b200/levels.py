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


lib.bssn_mesh_generate_levels.argtypes = [C.c_int, C.POINTER(C.c_int32), C.POINTER(BssnLevelBox), C.c_double,
                                          C.c_double, C.POINTER(BssnBlockDesc), C.POINTER(C.c_int),
                                          C.POINTER(C.c_int64)]
lib.bssn_mesh_create_levels.argtypes = [C.POINTER(BssnBlockDesc), C.c_int, C.c_int, C.POINTER(C.c_int32),
                                        C.POINTER(BssnLevelBox), C.POINTER(C.c_void_p)]
lib.bssn_mesh_levels_sync.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p]
lib.bssn_levels_maps.argtypes = [C.POINTER(BssnBlockDesc), C.c_int, C.c_int, C.POINTER(C.c_int32),
                                 C.POINTER(BssnLevelBox), C.POINTER(C.c_int64)] + [C.c_void_p] * 5


@dataclass
class LevelMeshSpec(MeshSpec):
    """A MeshSpec whose zipped state spans several level grids.  `h` is the
    finest spacing (the time step's), `h0` level 0's; G = (n_nodes, 1, 1)."""
    M0: tuple = (1, 1, 1)
    boxes: list = field(default_factory=list)   # [(lo, n)] per level, level octants
    h0: float = 0.0

    @property
    def nlevels(self):
        return len(self.boxes)

    def c_boxes(self):
        arr = (BssnLevelBox * self.nlevels)()
        for l, (lo, n) in enumerate(self.boxes):
            arr[l].lo[:] = list(lo)
            arr[l].n[:] = list(n)
        return arr

    def grids(self):
        """Per level: dict(lo, n, dims, offset, h, origin) of its node grid."""
        out, off = [], 0
        for l, (lo, n) in enumerate(self.boxes):
            dims = tuple(OCT * int(x) + 1 for x in n)
            h = self.h0 / 2 ** l
            origin = tuple(self.xmin + OCT * int(lo[d]) * h for d in range(3))
            out.append(dict(lo=tuple(lo), n=tuple(n), dims=dims, offset=off, h=h, origin=origin))
            off += dims[0] * dims[1] * dims[2]
        return out


def generate_levels(M0, boxes, xmin=-8.0, L=16.0):
    """Level 0 = the domain [xmin, xmin + L]^3 in M0 octants per axis; boxes
    = [(lo, n)] of levels 1.. in their own octants."""
    allb = [((0, 0, 0), tuple(M0))] + [(tuple(lo), tuple(n)) for lo, n in boxes]
    h0 = L / (OCT * M0[0])
    spec = LevelMeshSpec(None, 0, (0, 1, 1), h0 / 2 ** (len(allb) - 1), xmin, None, None,
                         tuple(M0), allb, h0)
    cb = spec.c_boxes()
    M = (C.c_int32 * 3)(*M0)
    n = C.c_int(0)
    nn = C.c_int64(0)
    check(lib.bssn_mesh_generate_levels(len(allb), M, cb, xmin, h0, None, C.byref(n), C.byref(nn)),
          "mesh_generate_levels")
    blocks = (BssnBlockDesc * n.value)()
    check(lib.bssn_mesh_generate_levels(len(allb), M, cb, xmin, h0, blocks, C.byref(n), C.byref(nn)),
          "mesh_generate_levels")
    spec.blocks, spec.nblocks = blocks, n.value
    spec.G = (int(nn.value), 1, 1)
    spec.sides = np.array([blocks[b].sz for b in range(n.value)], dtype=np.int32)
    return spec


def create_mesh_handle(spec: LevelMeshSpec):
    h = C.c_void_p()
    M = (C.c_int32 * 3)(*spec.M0)
    check(lib.bssn_mesh_create_levels(spec.blocks, spec.nblocks, spec.nlevels, M, spec.c_boxes(), C.byref(h)),
          "mesh_create_levels")
    return h


def _rows(U, off=0):
    n = U.shape[1]
    return (C.c_void_p * NVARS)(*[U.data_ptr() + (v * n + off) * 8 for v in range(NVARS)])


def sync(mesh, U, stream=None):
    """Level sync of the zipped state U ((24, n_nodes) CUDA tensor)."""
    check(lib.bssn_mesh_levels_sync(mesh.h, _rows(U), NVARS, stream_ptr(stream)), "mesh_levels_sync")


def initial_data_levels(U, spec: LevelMeshSpec, mesh=None, bh=(1.0, 0.0, 0.0, -1.0, 0.0, 0.0), m1=0.5,
                        m2=0.5, chi_floor=1e-4, eps=1e-8, seed=20261203, stream=None):
    """Brill-Lindquist data on every level grid (noise seed + level), then
    the level sync when a mesh handle is given."""
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
    cb = spec.c_boxes()
    sizes = (C.c_int64 * 5)()
    check(lib.bssn_levels_maps(spec.blocks, spec.nblocks, spec.nlevels, M, cb, sizes, None, None, None, None,
                               None), "levels_maps")
    npad, nn, ninj, npro, nint = [int(x) for x in sizes]
    unz = np.zeros(npad, dtype=np.int64)
    zp = np.zeros(nn, dtype=np.int64)
    inj = np.zeros((max(ninj, 1), 2), dtype=np.int64)
    pro = np.zeros((max(npro, 1), 2), dtype=np.int64)
    itp = np.zeros((max(nint, 1), 7), dtype=np.int64)
    check(lib.bssn_levels_maps(spec.blocks, spec.nblocks, spec.nlevels, M, cb, sizes, unz.ctypes.data,
                               zp.ctypes.data, inj.ctypes.data, pro.ctypes.data, itp.ctypes.data), "levels_maps")
    return dict(unzip_src=unz, zip_src=zp, inject=inj[:ninj], prolong=pro[:npro], interp=itp[:nint])
