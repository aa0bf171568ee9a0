"""ctypes access to the CPU oracles (test infrastructure only).

liboracle.so  -- this repository's CPU restatement (oracle/bssn_oracle.cpp)
libbssn_ref.so -- the reference's own stencils and generated equations,
                  compiled from the reference sources in place (oracle/_ref)
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
ORACLE_SO = os.path.join(ORACLE_DIR, "liboracle.so")
REF_SO = os.path.join(ORACLE_DIR, "_ref", "libbssn_ref.so")
NVARS = 24
_dp = C.POINTER(C.c_double)
_PA = C.c_void_p * NVARS


def build_oracle():
    if not os.path.exists(ORACLE_SO) or os.path.getmtime(ORACLE_SO) < os.path.getmtime(
            os.path.join(ORACLE_DIR, "bssn_oracle.cpp")):
        subprocess.run(["make", "-C", ORACLE_DIR, "liboracle.so"], check=True,
                       stdout=subprocess.DEVNULL)


class OrcParams(C.Structure):
    _fields_ = [("ko_sigma", C.c_double), ("lambda_", C.c_uint * 4),
                ("lambda_f", C.c_double * 2), ("eta_central", C.c_double),
                ("eta_outer", C.c_double), ("eta_width", C.c_double),
                ("cako_enabled", C.c_int), ("eps_cako_gauge", C.c_double),
                ("eps_cako_other", C.c_double)]


def params(ko_sigma=0.4, eta=2.0, cako=False, lam=(1, 1, 1, 1), lam_f=(1.0, 0.0),
           eta_outer=None, eta_width=40.0):
    """The oracle's parameter block (BSSN_GR/src/parameters.h names:
    BSSN_KO_SIGMA, BSSN_LAMBDA, BSSN_LAMBDA_F, RIT_ETA_CENTRAL / OUTER /
    WIDTH, BSSN_CAKO_ENABLED with the epsilons 0.99 / 0.3)."""
    outer = eta if eta_outer is None else eta_outer
    return OrcParams(ko_sigma, tuple(lam), tuple(lam_f), eta, outer, eta_width, int(cako), 0.99, 0.3)


# Parameter sets beyond the workloads' defaults: r-dependent eta, CAKO
# dissipation, gauge switches (lambda) and an alpha-dependent beta driver.
PARAM_SETS = {
    "default": {},
    "eta_r": dict(ko_sigma=0.1, eta=2.0, eta_outer=0.5, eta_width=3.0),
    "cako_lambda": dict(cako=True, lam=(1, 0, 1, 0), lam_f=(1.0, 0.5)),
}


def device_params(name, chi_floor=1e-4):
    """The same set as the library's BssnParams (CHI_FLOOR added)."""
    import bssn_b200 as B
    o = params(**PARAM_SETS[name])
    return B.BssnParams(o.ko_sigma, tuple(o.lambda_), tuple(o.lambda_f), o.eta_central, o.eta_outer,
                        o.eta_width, o.cako_enabled, o.eps_cako_gauge, o.eps_cako_other, chi_floor)


def P(a):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_dp)


def rows(a):
    """24 row pointers of a (24, n) float64 array."""
    assert a.flags.c_contiguous and a.shape[0] == NVARS
    return _PA(*[a.ctypes.data + v * a.shape[1] * 8 for v in range(NVARS)])


class Oracle:
    STENCILS = ["deriv644_x", "deriv644_y", "deriv644_z", "deriv644_xx", "deriv644_yy",
                "deriv644_zz", "ko_deriv42_x", "ko_deriv42_y", "ko_deriv42_z"]

    def __init__(self, path=ORACLE_SO, prefix="orc_"):
        self.lib = C.CDLL(path)
        self.prefix = prefix

    def stencil(self, kind, u, h, sz, bflag):
        out = np.zeros(int(np.prod(sz)))
        s = (C.c_uint * 3)(*sz)
        getattr(self.lib, self.prefix + self.STENCILS[kind])(P(out), P(u), C.c_double(h), s, C.c_uint(bflag))
        return out

    def bssnrhs(self, U, offset, pmin, pmax, side, bflag, prm):
        """RHS of one block; U is (24, n) with the block at `offset`."""
        R = np.zeros_like(U)
        n = side ** 3
        ws = np.zeros(288 * n) if self.prefix == "orc_" else np.zeros(138 * n)
        pm = np.ascontiguousarray(pmin, dtype=np.float64)
        px = np.ascontiguousarray(pmax, dtype=np.float64)
        sz = (C.c_uint * 3)(side, side, side)
        getattr(self.lib, self.prefix + "bssnrhs")(rows(R), rows(U), C.c_uint(offset), P(pm), P(px), sz,
                                                   C.c_uint(bflag), C.byref(prm), P(ws))
        return R

    def enforce(self, U, chi_floor=1e-4):
        """enforce_bssn_constraints on every column of a (24, n) array, in
        place; returns the number of violating nodes."""
        self.lib.orc_enforce.restype = C.c_int64
        return self.lib.orc_enforce(rows(U), C.c_int64(U.shape[1]), C.c_double(chi_floor))


def oracle():
    build_oracle()
    return Oracle()


class OrcBlock(C.Structure):
    _fields_ = [("offset", C.c_int64), ("sz", C.c_int32), ("bflag", C.c_uint32),
                ("g0", C.c_int32 * 3), ("level", C.c_int32),
                ("ptmin", C.c_double * 3), ("ptmax", C.c_double * 3)]


class OracleMeshSpec:
    """A workload mesh built by the oracle's own generator (no product
    library involved): the same attributes MeshOracle reads from the
    library's MeshSpec."""

    def __init__(self, mode, dims, p=(0.7, 0.2, 0.08, 0.02), seed=0, xmin=-8.0, L=16.0, lib=None,
                 origin=None):
        lib = (lib or oracle()).lib
        d = (C.c_int32 * 3)(*dims)
        pp = (C.c_double * 4)(*p)
        n = C.c_int(0)
        G = (C.c_int32 * 3)()
        h = C.c_double(0)
        lib.orc_mesh_generate.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_uint64, C.c_double,
                                          C.c_double, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        for blocks in (None, True):
            if blocks:
                blocks = (OrcBlock * n.value)()
            rc = lib.orc_mesh_generate(mode, d, pp, seed, xmin, L, blocks, C.byref(n), G, C.byref(h))
            assert rc == 0, rc
        if origin is not None:  # node (0,0,0) at origin per axis, the generator's corner formula
            for b in range(n.value):
                for k in range(3):
                    blocks[b].ptmin[k] = origin[k] + float(blocks[b].g0[k] - 3) * h.value
                    blocks[b].ptmax[k] = origin[k] + float(blocks[b].g0[k] - 3 + blocks[b].sz - 1) * h.value
            xmin = float(origin[0])
        self.origin = tuple(origin) if origin is not None else None
        self.blocks, self.nblocks = blocks, n.value
        self.G, self.h, self.xmin = tuple(G), h.value, xmin
        self.sides = np.array([blocks[b].sz for b in range(n.value)], dtype=np.int32)

    @property
    def origin3(self):
        return self.origin if self.origin is not None else (self.xmin,) * 3

    @property
    def n_nodes(self):
        return int(self.G[0]) * int(self.G[1]) * int(self.G[2])

    @property
    def n_unzip(self):
        b = self.blocks[self.nblocks - 1]
        return int(b.offset) + int(b.sz) ** 3

    def zones(self):
        return int(sum((int(s) - 6) ** 3 for s in self.sides))


def reference():
    if not os.path.exists(REF_SO):
        return None
    return Oracle(REF_SO, prefix="ref_")


def blocks_array(spec):
    """Mesh blocks as a ctypes array usable by the oracle (same layout as
    OrcBlock)."""
    return spec.blocks


class MeshOracle:
    """Oracle-side unzip / zip / RHS over a block list."""

    def __init__(self, spec, lib=None):
        self.spec = spec
        self.lib = (lib or oracle()).lib
        self.G = (C.c_int32 * 3)(*spec.G)

    def unzip(self, Z, nvars=NVARS):
        U = np.zeros((NVARS, self.spec.n_unzip))
        self.lib.orc_unzip(rows(U), rows(Z), self.spec.blocks, self.spec.nblocks, self.G, nvars)
        return U

    def zip(self, U, nvars=NVARS):
        Z = np.zeros((NVARS, self.spec.n_nodes))
        self.lib.orc_zip(rows(Z), rows(U), self.spec.blocks, self.spec.nblocks, self.G, nvars)
        return Z

    def unzip_map(self):
        m = np.zeros(self.spec.n_unzip, dtype=np.int64)
        self.lib.orc_unzip_map(m.ctypes.data_as(C.c_void_p), self.spec.blocks, self.spec.nblocks, self.G)
        return m

    def rhs(self, U, prm, nthreads=0):
        R = np.zeros_like(U)
        self.lib.orc_bssnRHS(rows(R), rows(U), self.spec.blocks, self.spec.nblocks, C.byref(prm), nthreads)
        return R

    def initial_data(self, bh=(1.0, 0.0, 0.0, -1.0, 0.0, 0.0), m1=0.5, m2=0.5, chi_floor=1e-4,
                     eps=1e-8, seed=20261203):
        Z = np.zeros((NVARS, self.spec.n_nodes))
        org = getattr(self.spec, "origin3", (self.spec.xmin,) * 3)
        xm = (C.c_double * 3)(*org)
        b = (C.c_double * 6)(*bh)
        self.lib.orc_initial_data(rows(Z), self.G, xm, C.c_double(self.spec.h), b, C.c_double(m1),
                                  C.c_double(m2), C.c_double(chi_floor), C.c_double(eps),
                                  C.c_uint64(seed))
        return Z

    def rk4_workspace(self):
        self.lib.orc_rk4_ws_doubles.restype = C.c_int64
        n = self.lib.orc_rk4_ws_doubles(self.G, C.c_int64(self.spec.n_unzip))
        return np.zeros(n)

    def rk4_step_ws(self, Z, dt, prm, ws, rhs_fn=None, chi_floor=1e-4, enforce_stages=True,
                    nthreads=0):
        """One RK4 step in a persistent workspace (rk4_workspace()); rhs_fn:
        the block-loop right-hand side (a ctypes function pointer, e.g. the
        reference's own ref_bssnRHS_blocks) or None for the oracle's."""
        self.lib.orc_rk4_step_ws.restype = C.c_int64
        self.lib.orc_rk4_step_ws.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_int64,
                                             C.c_double, C.c_void_p, C.c_double, C.c_int, C.c_int,
                                             C.c_void_p, C.c_void_p]
        fn = C.cast(rhs_fn, C.c_void_p) if rhs_fn is not None else None
        return self.lib.orc_rk4_step_ws(rows(Z), self.spec.blocks, self.spec.nblocks, self.G,
                                        self.spec.n_unzip, dt, C.byref(prm), chi_floor,
                                        int(enforce_stages), nthreads, fn, P(ws))

    def rk4_step_lowmem(self, Z, dt, prm, bufs, rhs_fn=None, chi_floor=1e-4, enforce_stages=True,
                        nthreads=0):
        """orc_rk4_step_lowmem: bufs = three (24, n_nodes) float64 arrays
        (accumulator, stage right-hand side, stage state)."""
        f = self.lib.orc_rk4_step_lowmem
        f.restype = C.c_int64
        f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_double, C.c_void_p, C.c_double,
                      C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        fn = C.cast(rhs_fn, C.c_void_p) if rhs_fn is not None else None
        return f(rows(Z), self.spec.blocks, self.spec.nblocks, self.G, dt, C.byref(prm), chi_floor,
                 int(enforce_stages), nthreads, fn, rows(bufs[0]), rows(bufs[1]), rows(bufs[2]))

    def rk4_step(self, Z, dt, prm, chi_floor=1e-4, enforce_stages=True, nthreads=0):
        self.lib.orc_rk4_step.restype = C.c_int64
        return self.lib.orc_rk4_step(rows(Z), self.spec.blocks, self.spec.nblocks, self.G,
                                     C.c_int64(self.spec.n_unzip), C.c_double(dt), C.byref(prm),
                                     C.c_double(chi_floor), int(enforce_stages), nthreads)


def interior_mask(spec):
    """Boolean mask over the unzipped vector selecting block interiors."""
    m = np.zeros(spec.n_unzip, dtype=bool)
    for b in range(spec.nblocks):
        blk = spec.blocks[b]
        s = int(blk.sz)
        cube = np.zeros((s, s, s), dtype=bool)
        cube[3:-3, 3:-3, 3:-3] = True
        m[int(blk.offset):int(blk.offset) + s ** 3] = cube.ravel()
    return m


def rel_err(ref, got):
    """Per-variable ||got - ref||_inf / ||ref||_inf (0 where ref is 0)."""
    num = np.abs(got - ref).max(axis=1)
    den = np.abs(ref).max(axis=1)
    return np.where(den > 0, num / np.where(den > 0, den, 1), num)


def oracle_constraints(spec, Uz, lib=None, threads=1):
    """ham, mom0..2 on every zipped node from the padded state Uz, by
    orc_physical_constraints per block (physcon.cpp:12-89 restated) and the
    oracle's zip; blocks spread over `threads` host threads (each block
    writes only its own interior)."""
    O = lib or oracle()
    Cz = np.zeros((NVARS, spec.n_unzip))
    rc, ru = rows(Cz), rows(Uz)

    def run(bs):
        ws = np.zeros(288 * 55 ** 3)
        for b in bs:
            blk = spec.blocks[b]
            s = int(blk.sz)
            pm = np.array(blk.ptmin[:])
            px = np.array(blk.ptmax[:])
            sz = (C.c_uint * 3)(s, s, s)
            O.lib.orc_physical_constraints(rc, ru, C.c_uint(int(blk.offset)), P(pm), P(px), sz,
                                           C.c_uint(int(blk.bflag)), P(ws))

    if threads <= 1:
        run(range(spec.nblocks))
    else:
        from concurrent.futures import ThreadPoolExecutor
        with ThreadPoolExecutor(threads) as ex:
            list(ex.map(run, [range(t, spec.nblocks, threads) for t in range(threads)]))
    return MeshOracle(spec, O).zip(Cz, nvars=4)[:4]


def constraint_norms_lowmem(spec, Z, lib=None, bh=(1.0, 0.0, 0.0, -1.0, 0.0, 0.0), radii=(0.5, 0.5),
                            threads=0):
    """The masked constraint L2 norms of a zipped state, block by block
    (orc_constraint_sums_lowmem: no unzipped copies)."""
    O = lib or oracle()
    f = O.lib.orc_constraint_sums_lowmem
    f.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                  C.c_void_p, C.c_void_p, C.c_int]
    sums = np.zeros(5)
    org = getattr(spec, "origin3", (spec.xmin,) * 3)
    f(rows(Z), spec.blocks, spec.nblocks, (C.c_int32 * 3)(*spec.G), (C.c_double * 3)(*org), spec.h,
      (C.c_double * 6)(*bh), (C.c_double * 2)(*radii), P(sums), threads)
    return np.sqrt(sums[:4] / sums[4])


def oracle_psi4(spec, Uz, lib=None):
    """psi4 (real, imaginary) on every zipped node from the padded state Uz,
    by orc_psi4 per block (pinned to the reference's physconeqs.cpp) and the
    oracle's zip."""
    O = lib or oracle()
    Cz = np.zeros((NVARS, spec.n_unzip))
    ws = np.zeros(288 * 55 ** 3)
    for b in range(spec.nblocks):
        blk = spec.blocks[b]
        s = int(blk.sz)
        pm = np.array(blk.ptmin[:])
        px = np.array(blk.ptmax[:])
        sz = (C.c_uint * 3)(s, s, s)
        O.lib.orc_psi4(P(Cz[0]), P(Cz[1]), rows(Uz), C.c_uint(int(blk.offset)), P(pm), P(px), sz,
                       C.c_uint(int(blk.bflag)), P(ws))
    return MeshOracle(spec, O).zip(Cz, nvars=2)[:2]


def l2_norms(spec, Cn, bh=(1.0, 0.0, 0.0, -1.0, 0.0, 0.0), radii=(0.5, 0.5)):
    """sqrt(sum c^2 / N) over nodes outside both puncture radii
    (grUtils.tcc:36-134)."""
    G = spec.G
    o = getattr(spec, "origin3", (spec.xmin,) * 3)
    g = np.arange(spec.n_nodes)
    x = o[0] + (g % G[0]) * spec.h
    y = o[1] + ((g // G[0]) % G[1]) * spec.h
    z = o[2] + (g // (G[0] * G[1])) * spec.h
    d1 = np.sqrt((x - bh[0]) ** 2 + (y - bh[1]) ** 2 + (z - bh[2]) ** 2)
    d2 = np.sqrt((x - bh[3]) ** 2 + (y - bh[4]) ** 2 + (z - bh[5]) ** 2)
    keep = ~((d1 < radii[0]) | (d2 < radii[1]))
    return np.sqrt((Cn[:, keep] ** 2).sum(axis=1) / keep.sum())
