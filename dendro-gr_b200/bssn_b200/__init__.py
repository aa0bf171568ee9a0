"""Python plumbing over the C ABI of libbssn_b200.so (include/bssn_b200.h).

PyTorch is used only to own device memory and streams; every computation is
a kernel of libbssn_b200.so.  Importing this module loads the library and
raises if it is missing: there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libbssn_b200.so")
NVARS = 24

VAR_NAMES = ["alpha", "chi", "K", "Gt0", "Gt1", "Gt2", "beta0", "beta1",
             "beta2", "B0", "B1", "B2", "gt0", "gt1", "gt2", "gt3", "gt4",
             "gt5", "At0", "At1", "At2", "At3", "At4", "At5"]

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `make -C dendro-gr_b200` "
        "(there is no CPU fallback)")
lib = C.CDLL(LIB_PATH)

_dp = C.POINTER(C.c_double)
_PtrArr = C.c_void_p * NVARS


class BssnParams(C.Structure):
    _fields_ = [("ko_sigma", C.c_double), ("lambda_", C.c_uint * 4),
                ("lambda_f", C.c_double * 2), ("eta_central", C.c_double),
                ("eta_outer", C.c_double), ("eta_width", C.c_double),
                ("cako_enabled", C.c_int), ("eps_cako_gauge", C.c_double),
                ("eps_cako_other", C.c_double), ("chi_floor", C.c_double)]


class BssnBlockDesc(C.Structure):
    _fields_ = [("offset", C.c_int64), ("sz", C.c_int32), ("bflag", C.c_uint32),
                ("g0", C.c_int32 * 3), ("level", C.c_int32),
                ("ptmin", C.c_double * 3), ("ptmax", C.c_double * 3)]


def default_params(ko_sigma=0.4, eta=2.0, chi_floor=1e-4, cako=False):
    """sigma=0.4, lambda={1,1,1,1}, lambda_f={1,0}, constant eta (RIT
    central = outer), CHI_FLOOR=1e-4: the workloads' parameters."""
    return BssnParams(ko_sigma, (1, 1, 1, 1), (1.0, 0.0), eta, eta, 40.0,
                      int(cako), 0.99, 0.3, chi_floor)


def _sig():
    vp, i, i64, d, u32 = C.c_void_p, C.c_int, C.c_int64, C.c_double, C.c_uint
    P = C.POINTER
    lib.bssn_version.restype = C.c_char_p
    lib.bssn_deriv644_f64.argtypes = [i, vp, vp, d, P(u32), u32, vp]
    lib.bssn_deriv644adv_f64.argtypes = [i, vp, vp, d, P(u32), vp, u32, vp]
    lib.bssn_bssnrhs_f64.argtypes = [vp, vp, i64, P(d), P(d), P(u32), u32, P(BssnParams), vp]
    lib.bssn_mesh_create.argtypes = [P(BssnBlockDesc), i, P(C.c_int32), P(vp)]
    lib.bssn_mesh_destroy.argtypes = [vp]
    lib.bssn_mesh_unzip_size.argtypes = [vp]
    lib.bssn_mesh_unzip_size.restype = i64
    lib.bssn_rhs_blocks_f64.argtypes = [vp, vp, vp, P(BssnParams), i, vp]
    lib.bssn_unzip_f64.argtypes = [vp, vp, vp, i, vp]
    lib.bssn_zip_f64.argtypes = [vp, vp, vp, i, vp]
    lib.bssn_rk4_stage_f64.argtypes = [i, vp, vp, vp, i64, d, i, d, vp, vp]
    lib.bssn_enforce_f64.argtypes = [vp, i64, d, vp, vp]
    lib.bssn_initial_data_f64.argtypes = [vp, P(C.c_int32), P(d), d, P(d), d, d, d, d, C.c_uint64, vp]
    lib.bssn_mesh_generate.argtypes = [i, P(C.c_int32), P(d), C.c_uint64, d, d,
                                       P(BssnBlockDesc), P(i), P(C.c_int32), P(d)]
    lib.bssn_rk4_plan_create.argtypes = [vp, P(BssnParams), i, P(vp)]
    lib.bssn_rk4_plan_step.argtypes = [vp, vp, d, vp]
    lib.bssn_rk4_plan_diagnostics.argtypes = [vp, vp, P(d), d, P(d), P(d), vp, vp]
    lib.bssn_rk4_plan_step_diag.argtypes = [vp, vp, d, P(d), d, P(d), P(d), vp, vp]
    lib.bssn_rk4_plan_diag_fields.argtypes = [vp, vp]
    lib.bssn_rk4_plan_copy_diag_fields.argtypes = [vp, vp, i, vp]
    lib.bssn_rk4_plan_autotune.argtypes = [vp, vp, i, vp, P(C.c_float)]
    lib.bssn_rk4_plan_tile.argtypes = [vp, i]
    lib.bssn_rk4_plan_set_tile.argtypes = [vp, i, i]
    lib.bssn_rk4_plan_time_kernels.argtypes = [vp, i, vp, P(d)]
    lib.bssn_rk4_plan_launches_per_step.argtypes = [vp]
    lib.bssn_tile_mode.argtypes = [i]
    lib.bssn_mesh_partition.argtypes = [P(BssnBlockDesc), i, i, P(C.c_int32)]
    lib.bssn_rk4_plan_stage.argtypes = [vp, vp, d, i, vp]
    lib.bssn_rk4_plan_stage_state.argtypes = [vp, vp]
    lib.bssn_halo_pack_f64.argtypes = [vp, vp, vp, i64, vp]
    lib.bssn_halo_unpack_f64.argtypes = [vp, vp, vp, i64, vp]
    lib.bssn_rk4_plan_violations.argtypes = [vp, P(i)]
    lib.bssn_rk4_plan_destroy.argtypes = [vp]
    lib.bssn_constraints_f64.argtypes = [vp, vp, vp, vp]
    lib.bssn_constraint_norms_f64.argtypes = [vp, vp, i, P(d), d, P(d), P(d), vp, vp]
    lib.bssn_rk4_plan_time_rhs.argtypes = [vp, i, vp, P(C.c_float)]
    lib.bssn_fp64_probe.argtypes = [vp, i, vp, P(d)]
    lib.bssn_mesh_num_elements.argtypes = [vp]
    lib.bssn_mesh_num_elements.restype = i64
    lib.bssn_remesh_wavelet_f64.argtypes = [vp, vp, i, d, vp, vp, vp, vp]
    lib.bssn_remesh_features_f64.argtypes = [vp, vp, vp, vp]
    lib.bssn_remesh_mlp_fwd_bf16.argtypes = [vp, vp, vp, i, vp, vp]
    lib.bssn_remesh_mlp_fwd_fp32_bf16.argtypes = [vp, vp, vp, i, vp, vp]
    lib.bssn_remesh_mlp_grad_scratch.argtypes = [i]
    lib.bssn_remesh_mlp_grad_scratch.restype = C.c_size_t
    lib.bssn_remesh_mlp_bwd_bf16.argtypes = [vp, vp, vp, vp, vp, i, vp, vp, vp, vp]
    lib.bssn_remesh_mlp_step_bf16.argtypes = [vp, vp, vp, vp, vp, C.c_float, C.c_float, C.c_float,
                                              C.c_float, i, vp]
    lib.bssn_remesh_decide_work_bytes.argtypes = [vp]
    lib.bssn_remesh_decide_work_bytes.restype = C.c_size_t
    lib.bssn_remesh_decide_f64.argtypes = [vp, vp, vp, vp, C.c_float, C.c_float, d, C.c_uint64, d,
                                           vp, vp, vp, C.c_size_t, vp]
    lib.bssn_tile_count.argtypes = []
    lib.bssn_tile_info.argtypes = [i, P(i)]


_sig()


class BssnError(RuntimeError):
    pass


def check(rc, what=""):
    if rc != 0:
        raise BssnError(f"{what} failed with status {rc}")


def ptrs(t, n_per_var=None):
    """Array of 24 device pointers for a (24, n) float64 CUDA tensor (or a
    list of 24 tensors)."""
    if isinstance(t, (list, tuple)):
        return _PtrArr(*[x.data_ptr() for x in t])
    assert t.dtype.is_floating_point and t.is_cuda and t.is_contiguous()
    n = t.shape[-1] if n_per_var is None else n_per_var
    base = t.data_ptr()
    return _PtrArr(*[base + v * n * 8 for v in range(NVARS)])


def stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


# ---------------------------------------------------------------------------
# meshes
# ---------------------------------------------------------------------------
@dataclass
class MeshSpec:
    blocks: object          # ctypes array of BssnBlockDesc
    nblocks: int
    G: tuple
    h: float
    xmin: float
    sides: np.ndarray = field(default=None)
    # coordinate of node (0,0,0) per axis when it differs between axes (the
    # box of one rank of a partitioned mesh); None: xmin on every axis
    origin: tuple = None

    @property
    def origin3(self):
        return tuple(self.origin) if self.origin is not None else (self.xmin,) * 3

    @property
    def n_nodes(self):
        return int(self.G[0]) * int(self.G[1]) * int(self.G[2])

    @property
    def n_unzip(self):
        b = self.blocks[self.nblocks - 1]
        return int(b.offset) + int(b.sz) ** 3

    def zones(self):
        return int(sum((int(s) - 6) ** 3 for s in self.sides))

    def as_numpy(self):
        """Structured copy for the CPU oracle (same memory layout)."""
        return np.ctypeslib.as_array(self.blocks, shape=(self.nblocks,)).copy()


def generate_mesh(mode, dims, p=(0.7, 0.2, 0.08, 0.02), seed=0, xmin=-8.0, L=16.0, origin=None):
    """mode 0: uniform 13^3 blocks on a dims[0]^3 octant box; mode 1: seeded
    mix of 13/19/31/55 blocks on a dims super-cell box (8^3 octants each).
    The longest axis spans L; node (0,0,0) sits at xmin on every axis, or at
    `origin` (per axis) when given -- e.g. to centre a non-cubic box on the
    coordinate origin, where the Sommerfeld condition measures r from."""
    d = (C.c_int32 * 3)(*dims)
    pp = (C.c_double * 4)(*p)
    n = C.c_int(0)
    G = (C.c_int32 * 3)()
    h = C.c_double(0)
    check(lib.bssn_mesh_generate(mode, d, pp, seed, xmin, L, None, C.byref(n), G, C.byref(h)), "mesh_generate")
    blocks = (BssnBlockDesc * n.value)()
    check(lib.bssn_mesh_generate(mode, d, pp, seed, xmin, L, blocks, C.byref(n), G, C.byref(h)), "mesh_generate")
    sides = np.array([blocks[b].sz for b in range(n.value)], dtype=np.int32)
    if origin is not None:
        reorigin_blocks(blocks, n.value, origin, h.value)
        return MeshSpec(blocks, n.value, tuple(G), h.value, float(origin[0]), sides, tuple(origin))
    return MeshSpec(blocks, n.value, tuple(G), h.value, xmin, sides)


def reorigin_blocks(blocks, nblocks, origin, h):
    """Block corners for node (0,0,0) at `origin`: ptmin = origin + (g0 - 3) h,
    ptmax = origin + (g0 - 3 + s - 1) h per axis (the generator's formula)."""
    for b in range(nblocks):
        blk = blocks[b]
        for k in range(3):
            blk.ptmin[k] = origin[k] + float(blk.g0[k] - 3) * h
            blk.ptmax[k] = origin[k] + float(blk.g0[k] - 3 + blk.sz - 1) * h


class Mesh:
    """Device mesh handle (bssn_mesh)."""

    def __init__(self, spec: MeshSpec):
        self.spec = spec
        self.h = C.c_void_p()
        if getattr(spec, "boxes", None) or getattr(spec, "patches", None):  # multi-level mesh (levels.py)
            from .levels import create_mesh_handle
            self.h = create_mesh_handle(spec)
        else:
            G = (C.c_int32 * 3)(*spec.G)
            check(lib.bssn_mesh_create(spec.blocks, spec.nblocks, G, C.byref(self.h)), "mesh_create")
        self.n_unzip = lib.bssn_mesh_unzip_size(self.h)

    def close(self):
        if self.h:
            lib.bssn_mesh_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def unzip(self, unz, zip_, nvars=NVARS, stream=None):
        check(lib.bssn_unzip_f64(self.h, ptrs(unz), ptrs(zip_), nvars, stream_ptr(stream)), "unzip")

    def zip(self, zip_, unz, nvars=NVARS, stream=None):
        check(lib.bssn_zip_f64(self.h, ptrs(zip_), ptrs(unz), nvars, stream_ptr(stream)), "zip")

    def rhs(self, out, u, params, tile=-1, stream=None):
        check(lib.bssn_rhs_blocks_f64(self.h, ptrs(out), ptrs(u), C.byref(params), tile, stream_ptr(stream)), "rhs_blocks")


def bssnrhs_block(out, u, offset, pmin, pmax, side, bflag, params, stream=None):
    pm = (C.c_double * 3)(*pmin)
    px = (C.c_double * 3)(*pmax)
    sz = (C.c_uint * 3)(side, side, side)
    check(lib.bssn_bssnrhs_f64(ptrs(out), ptrs(u), offset, pm, px, sz, bflag, C.byref(params), stream_ptr(stream)), "bssnrhs")


def deriv(kind, D, u, h, sz, bflag, stream=None):
    s = (C.c_uint * 3)(*sz)
    check(lib.bssn_deriv644_f64(kind, C.c_void_p(D.data_ptr()), C.c_void_p(u.data_ptr()), h, s, bflag, stream_ptr(stream)), "deriv644")


def initial_data(U, spec: MeshSpec, bh=(1.0, 0.0, 0.0, -1.0, 0.0, 0.0), m1=0.5, m2=0.5,
                 chi_floor=1e-4, eps=1e-8, seed=20261203, stream=None):
    G = (C.c_int32 * 3)(*spec.G)
    xm = (C.c_double * 3)(*spec.origin3)
    b = (C.c_double * 6)(*bh)
    check(lib.bssn_initial_data_f64(ptrs(U), G, xm, spec.h, b, m1, m2, chi_floor, eps, seed, stream_ptr(stream)), "initial_data")


def rk4_stage(stage, out, prev, k, n, dt, enforce=True, chi_floor=1e-4, status=None, stream=None):
    if stage < 3:
        kp = ptrs(k)
    else:
        kp = (C.c_void_p * (4 * NVARS))(*[p for kk in k for p in ptrs(kk)])
    st = C.c_void_p(status.data_ptr()) if status is not None else None
    check(lib.bssn_rk4_stage_f64(stage, ptrs(out), ptrs(prev), kp, n, dt, int(enforce), chi_floor, st, stream_ptr(stream)), "rk4_stage")


def enforce(U, n, chi_floor=1e-4, status=None, stream=None):
    st = C.c_void_p(status.data_ptr()) if status is not None else None
    check(lib.bssn_enforce_f64(ptrs(U), n, chi_floor, st, stream_ptr(stream)), "enforce")


class PlainRK4:
    """The plain GPU path of one classical RK4 step, mirroring
    BSSN_GR/src/rkBSSN.cpp:764-860 call for call: per stage unzip -> bssnRHS
    over all blocks -> zip -> stage axpy (+ enforce)."""

    def __init__(self, mesh: Mesh, params, enforce_stages=True, tile=-1):
        import torch
        self.mesh = mesh
        self.params = params
        self.enforce_stages = enforce_stages
        self.tile = tile
        n = mesh.spec.n_nodes
        nu = mesh.n_unzip
        dev = "cuda"
        self.prev = torch.empty((NVARS, n), dtype=torch.float64, device=dev)
        self.im = torch.empty((NVARS, n), dtype=torch.float64, device=dev)
        self.k = [torch.empty((NVARS, n), dtype=torch.float64, device=dev) for _ in range(4)]
        self.uz = torch.zeros((NVARS, nu), dtype=torch.float64, device=dev)
        self.rz = torch.zeros((NVARS, nu), dtype=torch.float64, device=dev)
        self.status = torch.zeros(1, dtype=torch.int32, device=dev)

    def step(self, U, dt, stream=None):
        n = self.mesh.spec.n_nodes
        cf = self.params.chi_floor
        self.prev.copy_(U)
        for stage in range(4):
            src = U if stage == 0 else self.im
            self.mesh.unzip(self.uz, src, stream=stream)
            self.mesh.rhs(self.rz, self.uz, self.params, tile=self.tile, stream=stream)
            self.mesh.zip(self.k[stage], self.rz, stream=stream)
            if stage < 3:
                rk4_stage(stage, self.im, self.prev, self.k[stage], n, dt,
                          self.enforce_stages, cf, self.status, stream)
            else:
                rk4_stage(3, U, self.prev, self.k, n, dt, True, cf, self.status, stream)


def tiles():
    """(bx, by, bz, threads) per tile id."""
    out = []
    info = (C.c_int * 4)()
    for t in range(lib.bssn_tile_count()):
        check(lib.bssn_tile_info(t, info), "tile_info")
        out.append(tuple(info))
    return out


def tile_mode(t):
    """0: fused kernel; 1: split derivative + equation passes."""
    return lib.bssn_tile_mode(t)


PLAN_ENFORCE_STAGES = 1
PLAN_GRAPH = 2
PLAN_PER_BLOCK = 4
PLAN_DIRECT = 8
PLAN_DIAG_PSI4 = 16


class RK4Plan:
    """bssn_rk4_plan: one whole RK4 step (unzip -> fused RHS -> zip+stage
    update, x4), batched per block-size bucket and optionally captured as a
    CUDA graph; or the plain path with one RHS launch per block."""

    def __init__(self, mesh: Mesh, params, flags=PLAN_ENFORCE_STAGES | PLAN_GRAPH):
        self.mesh = mesh
        self.params = params
        self.h = C.c_void_p()
        check(lib.bssn_rk4_plan_create(mesh.h, C.byref(params), flags, C.byref(self.h)), "rk4_plan_create")

    def step(self, U, dt, stream=None):
        check(lib.bssn_rk4_plan_step(self.h, ptrs(U), dt, stream_ptr(stream)), "rk4_plan_step")

    def _diag_args(self, norms, bh, radii):
        spec = self.mesh.spec
        assert norms.is_cuda and norms.dtype.is_floating_point and norms.numel() >= 4
        return ((C.c_double * 3)(*spec.origin3), spec.h, (C.c_double * 6)(*bh),
                (C.c_double * 2)(*radii), C.c_void_p(norms.data_ptr()))

    def diagnostics(self, U, norms, bh=(1.0, 0.0, 0.0, -1.0, 0.0, 0.0), radii=(0.5, 0.5), stream=None):
        """Masked L2 norms of ham, mom0..2 of the state U into the CUDA
        tensor `norms` (4 doubles), on the device."""
        xm, h, b, r, nd = self._diag_args(norms, bh, radii)
        check(lib.bssn_rk4_plan_diagnostics(self.h, ptrs(U), xm, h, b, r, nd, stream_ptr(stream)),
              "rk4_plan_diagnostics")

    def step_diag(self, U, dt, norms, bh=(1.0, 0.0, 0.0, -1.0, 0.0, 0.0), radii=(0.5, 0.5),
                  stream=None):
        """One step, then the constraint norms of the new state into `norms`
        (one graph with PLAN_GRAPH)."""
        xm, h, b, r, nd = self._diag_args(norms, bh, radii)
        check(lib.bssn_rk4_plan_step_diag(self.h, ptrs(U), dt, xm, h, b, r, nd, stream_ptr(stream)),
              "rk4_plan_step_diag")

    def diag_fields(self, out, stream=None):
        """Copy the plan's diagnostic fields into `out` ((4 or 6, n_nodes)
        float64 CUDA tensor): ham, mom0..2 and, with PLAN_DIAG_PSI4, psi4
        real and imaginary, as written by the last diagnostics call."""
        nf = out.shape[0]
        dst = (C.c_void_p * nf)(*[out[c].data_ptr() for c in range(nf)])
        check(lib.bssn_rk4_plan_copy_diag_fields(self.h, dst, nf, stream_ptr(stream)), "copy_diag_fields")
        return out

    def autotune(self, U, reps=3, stream=None):
        sides = sorted(set(self.mesh.spec.sides.tolist()))
        nt = lib.bssn_tile_count()
        times = (C.c_float * (len(sides) * nt))()
        check(lib.bssn_rk4_plan_autotune(self.h, ptrs(U), reps, stream_ptr(stream), times), "autotune")
        table = {side: [times[i * nt + t] for t in range(nt)] for i, side in enumerate(sides)}
        chosen = {side: lib.bssn_rk4_plan_tile(self.h, side) for side in sides}
        return chosen, table

    def set_tile(self, tile, side=0):
        """Pin a tile (for every side when side is 0) instead of autotuning."""
        check(lib.bssn_rk4_plan_set_tile(self.h, side, tile), "set_tile")
        sides = sorted(set(self.mesh.spec.sides.tolist()))
        return {sd: lib.bssn_rk4_plan_tile(self.h, sd) for sd in sides}

    def violations(self):
        c = C.c_int(0)
        check(lib.bssn_rk4_plan_violations(self.h, C.byref(c)), "violations")
        return c.value

    def close(self):
        if self.h:
            lib.bssn_rk4_plan_destroy(self.h)
            self.h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _cons_ptrs(cons):
    assert cons.is_cuda and cons.dtype.is_floating_point and cons.is_contiguous()
    return (C.c_void_p * 4)(*[cons.data_ptr() + c * cons.shape[1] * 8 for c in range(4)])


def constraints(mesh: Mesh, cons, unz, stream=None):
    """ham, mom0..2 of the padded stage state `unz` into the zipped (4, n)
    tensor `cons` (owned nodes)."""
    check(lib.bssn_constraints_f64(mesh.h, ptrs(unz), _cons_ptrs(cons), stream_ptr(stream)), "constraints")


def constraint_norms(mesh: Mesh, cons, norms, bh=(1.0, 0.0, 0.0, -1.0, 0.0, 0.0),
                     radii=(0.5, 0.5), ncons=4, stream=None):
    """Masked L2 norms sqrt(sum c^2 / N) of the 4 zipped constraint fields
    into the CUDA tensor `norms` (>= ncons doubles)."""
    spec = mesh.spec
    xm = (C.c_double * 3)(*spec.origin3)
    b = (C.c_double * 6)(*bh)
    r = (C.c_double * 2)(*radii)
    check(lib.bssn_constraint_norms_f64(mesh.h, _cons_ptrs(cons), ncons, xm, spec.h, b, r,
                                        C.c_void_p(norms.data_ptr()), stream_ptr(stream)),
          "constraint_norms")


# ---------------------------------------------------------------------------
# remesh indicator
# ---------------------------------------------------------------------------
MLP_NPARAM = 5313


def _vp(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def wavelet_scores(mesh: Mesh, unz, tol=1e-6, nvars=NVARS, stream=None):
    """Exact wavelet test: (scores[num_elements, nvars], ratio[nblocks],
    flags[nblocks]) as CUDA tensors."""
    import torch
    ne = lib.bssn_mesh_num_elements(mesh.h)
    nb = mesh.spec.nblocks
    scores = torch.empty((ne, nvars), dtype=torch.float64, device="cuda")
    ratio = torch.empty(nb, dtype=torch.float64, device="cuda")
    flags = torch.empty(nb, dtype=torch.uint8, device="cuda")
    check(lib.bssn_remesh_wavelet_f64(mesh.h, ptrs(unz), nvars, tol, _vp(scores), _vp(ratio), _vp(flags),
                                      stream_ptr(stream)), "remesh_wavelet")
    return scores, ratio, flags


def block_features(mesh: Mesh, unz, stream=None):
    import torch
    f = torch.empty((mesh.spec.nblocks, 16), dtype=torch.float32, device="cuda")
    check(lib.bssn_remesh_features_f64(mesh.h, ptrs(unz), _vp(f), stream_ptr(stream)), "remesh_features")
    return f


class RemeshMLP:
    """The 16 -> 64 -> 64 -> 1 GELU indicator network: FP32 master
    parameters, BF16 compute copy, Adam state, input normalisation."""

    def __init__(self, seed=0):
        import torch
        g = torch.Generator().manual_seed(seed)
        p = torch.zeros(MLP_NPARAM, dtype=torch.float32)
        # He-style init of the weight blocks; biases zero
        p[0:1024] = torch.randn(1024, generator=g) * (2.0 / 16) ** 0.5
        p[1088:1088 + 4096] = torch.randn(4096, generator=g) * (2.0 / 64) ** 0.5
        p[5248:5312] = torch.randn(64, generator=g) * (1.0 / 64) ** 0.5
        self.master = p.cuda()
        self.wq = self.master.to(torch.bfloat16)
        self.m = torch.zeros_like(self.master)
        self.v = torch.zeros_like(self.master)
        self.norm = torch.cat([torch.zeros(16), torch.ones(16)]).cuda()
        self.t = 0
        self.lo, self.hi = 0.02, 0.98

    def set_norm(self, X):
        mu = X.mean(0)
        sd = X.std(0).clamp_min(1e-3)
        import torch
        self.norm = torch.cat([mu, 1.0 / sd]).float().contiguous()

    def logits(self, X, stream=None):
        """Logits of the decisions' forward (tensor cores, BF16 operands)."""
        import torch
        out = torch.empty(X.shape[0], dtype=torch.float32, device="cuda")
        check(lib.bssn_remesh_mlp_fwd_bf16(_vp(self.wq), _vp(self.norm), _vp(X), X.shape[0], _vp(out),
                                           stream_ptr(stream)), "mlp_fwd")
        return out

    def logits_fp32(self, X, stream=None):
        """Logits with FP32 activations (the training gradient's forward)."""
        import torch
        out = torch.empty(X.shape[0], dtype=torch.float32, device="cuda")
        check(lib.bssn_remesh_mlp_fwd_fp32_bf16(_vp(self.wq), _vp(self.norm), _vp(X), X.shape[0], _vp(out),
                                                stream_ptr(stream)), "mlp_fwd_fp32")
        return out

    def grad(self, X, Y, Cw=None, stream=None):
        import torch
        n = X.shape[0]
        scratch = torch.empty(lib.bssn_remesh_mlp_grad_scratch(n), dtype=torch.float32, device="cuda")
        g = torch.empty(MLP_NPARAM, dtype=torch.float32, device="cuda")
        loss = torch.empty(1, dtype=torch.float32, device="cuda")
        check(lib.bssn_remesh_mlp_bwd_bf16(_vp(self.wq), _vp(self.norm), _vp(X), _vp(Y), _vp(Cw), n,
                                           _vp(g), _vp(loss), _vp(scratch), stream_ptr(stream)), "mlp_bwd")
        return g, loss

    def step(self, g, lr=3e-3, b1=0.9, b2=0.999, eps=1e-8, stream=None):
        self.t += 1
        check(lib.bssn_remesh_mlp_step_bf16(_vp(self.master), _vp(self.wq), _vp(g), _vp(self.m), _vp(self.v),
                                            lr, b1, b2, eps, self.t, stream_ptr(stream)), "mlp_step")


def remesh_decide(mesh: Mesh, unz, net: RemeshMLP, tol=1e-6, audit_frac=0.05, seed=7, work=None,
                  stream=None):
    """Learned remesh flags with the exact-test fallback and audit; returns
    (flags uint8[nblocks], stats int32[4])."""
    import torch
    nb = mesh.spec.nblocks
    wb = lib.bssn_remesh_decide_work_bytes(mesh.h)
    if work is None or work.numel() < wb:
        work = torch.empty(wb, dtype=torch.uint8, device="cuda")
    flags = torch.empty(nb, dtype=torch.uint8, device="cuda")
    stats = torch.zeros(4, dtype=torch.int32, device="cuda")
    check(lib.bssn_remesh_decide_f64(mesh.h, ptrs(unz), _vp(net.wq), _vp(net.norm), net.lo, net.hi, audit_frac,
                                     seed, tol, _vp(flags), _vp(stats), _vp(work), wb, stream_ptr(stream)),
          "remesh_decide")
    return flags, stats


lib.bssn_remesh_decide2_elem_work_bytes.argtypes = [C.c_void_p]
lib.bssn_remesh_decide2_elem_work_bytes.restype = C.c_size_t
lib.bssn_remesh_decide2_elem_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float,
                                             C.c_float, C.c_void_p, C.c_void_p, C.c_float, C.c_float,
                                             C.c_double, C.c_uint64, C.c_double, C.c_double, C.c_void_p,
                                             C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]
lib.bssn_remesh_element_features_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]


def element_features(mesh: Mesh, unz, stream=None):
    """16 features per element (num_elements x 16 float32, CUDA)."""
    import torch
    ne = lib.bssn_mesh_num_elements(mesh.h)
    f = torch.empty((ne, 16), dtype=torch.float32, device="cuda")
    check(lib.bssn_remesh_element_features_f64(mesh.h, ptrs(unz), _vp(f), stream_ptr(stream)),
          "remesh_element_features")
    return f


def remesh_decide2_elem(mesh: Mesh, unz, net_refine: RemeshMLP, net_keep: RemeshMLP, tol=1e-6, keep_fac=0.1,
                        audit_frac=0.05, seed=7, work=None, stream=None):
    """Block refine and keep flags from per-element decisions (networks
    trained on element features and labels): the exact test runs only on the
    elements either network is unsure of and on a seeded audit sample of the
    elements; a block takes a flag when any of its elements does.  Returns
    (refine uint8[nblocks], keep uint8[nblocks], stats int32[8] counted per
    element)."""
    import torch
    nb = mesh.spec.nblocks
    wb = lib.bssn_remesh_decide2_elem_work_bytes(mesh.h)
    if work is None or work.numel() < wb:
        work = torch.empty(wb, dtype=torch.uint8, device="cuda")
    refine = torch.empty(nb, dtype=torch.uint8, device="cuda")
    keep = torch.empty(nb, dtype=torch.uint8, device="cuda")
    stats = torch.zeros(8, dtype=torch.int32, device="cuda")
    check(lib.bssn_remesh_decide2_elem_f64(mesh.h, ptrs(unz), _vp(net_refine.wq), _vp(net_refine.norm),
                                           net_refine.lo, net_refine.hi, _vp(net_keep.wq), _vp(net_keep.norm),
                                           net_keep.lo, net_keep.hi, audit_frac, seed, tol, keep_fac, _vp(refine),
                                           _vp(keep), _vp(stats), _vp(work), wb, stream_ptr(stream)),
          "remesh_decide2_elem")
    return refine, keep, stats


lib.bssn_remesh_decide2_work_bytes.argtypes = [C.c_void_p]
lib.bssn_remesh_decide2_work_bytes.restype = C.c_size_t
lib.bssn_remesh_decide2_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_float,
                                        C.c_float, C.c_void_p, C.c_void_p, C.c_float, C.c_float,
                                        C.c_double, C.c_uint64, C.c_double, C.c_double, C.c_void_p,
                                        C.c_void_p, C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p]


def remesh_decide2(mesh: Mesh, unz, net_refine: RemeshMLP, net_keep: RemeshMLP, tol=1e-6, keep_fac=0.1,
                   audit_frac=0.05, seed=7, work=None, stream=None):
    """Refine and keep flags (exact: block score above tol / above
    keep_fac * tol) learned in one pass: one feature pass, both networks, one
    exact-test pass over the blocks either network is unsure of and one
    audit sample.  Returns (refine uint8[nblocks], keep uint8[nblocks],
    stats int32[8])."""
    import torch
    nb = mesh.spec.nblocks
    wb = lib.bssn_remesh_decide2_work_bytes(mesh.h)
    if work is None or work.numel() < wb:
        work = torch.empty(wb, dtype=torch.uint8, device="cuda")
    refine = torch.empty(nb, dtype=torch.uint8, device="cuda")
    keep = torch.empty(nb, dtype=torch.uint8, device="cuda")
    stats = torch.zeros(8, dtype=torch.int32, device="cuda")
    check(lib.bssn_remesh_decide2_f64(mesh.h, ptrs(unz), _vp(net_refine.wq), _vp(net_refine.norm), net_refine.lo,
                                      net_refine.hi, _vp(net_keep.wq), _vp(net_keep.norm), net_keep.lo,
                                      net_keep.hi, audit_frac, seed, tol, keep_fac, _vp(refine), _vp(keep),
                                      _vp(stats), _vp(work), wb, stream_ptr(stream)), "remesh_decide2")
    return refine, keep, stats
