"""Error behaviour of the C ABI: every entry point returns a status code for
bad arguments (null pointers, unknown kinds, block sizes outside
{13,19,31,55}, out-of-range stages, sizes beyond a documented limit) before
it touches a device -- no trap, no exit (the reference exits or asserts).
Runs on the CPU: the placeholder pointers are never dereferenced."""
import ctypes as C

import pytest

import bssn_b200 as B

lib = B.lib
EINVAL, EBLOCKSIZE, EKIND, ELIMIT = 1, 2, 3, 6
FAKE = C.c_void_p(0x1000)
PTRS = (C.c_void_p * 24)(*([0x1000] * 24))


def sz(a, b, c):
    return (C.c_uint * 3)(a, b, c)


def test_stencil_arguments():
    lib.bssn_deriv644_f64.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p, C.c_uint, C.c_void_p]
    assert lib.bssn_deriv644_f64(0, None, FAKE, 0.1, sz(13, 13, 13), 0, None) == EINVAL
    assert lib.bssn_deriv644_f64(9, FAKE, FAKE, 0.1, sz(13, 13, 13), 0, None) == EKIND
    assert lib.bssn_deriv644_f64(-1, FAKE, FAKE, 0.1, sz(13, 13, 13), 0, None) == EKIND
    assert lib.bssn_deriv644_f64(0, FAKE, FAKE, 0.1, sz(11, 13, 13), 0, None) == EBLOCKSIZE
    lib.bssn_deriv644adv_f64.argtypes = [C.c_int, C.c_void_p, C.c_void_p, C.c_double, C.c_void_p,
                                         C.c_void_p, C.c_uint, C.c_void_p]
    assert lib.bssn_deriv644adv_f64(3, FAKE, FAKE, 0.1, sz(13, 13, 13), FAKE, 0, None) == EKIND


def test_block_rhs_arguments():
    pm = (C.c_double * 3)(0, 0, 0)
    prm = B.default_params()
    f = lib.bssn_bssnrhs_f64
    assert f(None, PTRS, 0, pm, pm, sz(13, 13, 13), 0, C.byref(prm), None) == EINVAL
    assert f(PTRS, PTRS, 0, pm, pm, sz(13, 13, 13), 0, None, None) == EINVAL
    assert f(PTRS, PTRS, 0, pm, pm, sz(13, 13, 19), 0, C.byref(prm), None) == EBLOCKSIZE
    assert f(PTRS, PTRS, 0, pm, pm, sz(14, 14, 14), 0, C.byref(prm), None) == EBLOCKSIZE


def test_mesh_and_plan_handles():
    G = (C.c_int32 * 3)(25, 25, 25)
    out = C.c_void_p()
    assert lib.bssn_mesh_create(None, 1, G, C.byref(out)) == EINVAL
    blocks = (B.BssnBlockDesc * 1)()
    assert lib.bssn_mesh_create(blocks, 0, G, C.byref(out)) == EINVAL
    assert lib.bssn_mesh_destroy(None) == EINVAL
    lib.bssn_mesh_unzip_size.restype = C.c_int64
    assert lib.bssn_mesh_unzip_size(None) == -1
    prm = B.default_params()
    assert lib.bssn_rhs_blocks_f64(None, PTRS, PTRS, C.byref(prm), -1, None) == EINVAL
    assert lib.bssn_unzip_f64(None, PTRS, PTRS, 25, None) == EINVAL
    assert lib.bssn_zip_f64(None, PTRS, PTRS, 0, None) == EINVAL
    assert lib.bssn_rk4_plan_create(None, C.byref(prm), 0, C.byref(out)) == EINVAL
    assert lib.bssn_rk4_plan_step(None, PTRS, C.c_double(0.1), None) == EINVAL
    assert lib.bssn_rk4_plan_stage(None, PTRS, 0.1, 0, None) == EINVAL
    assert lib.bssn_rk4_plan_stage(FAKE, PTRS, 0.1, 4, None) == EINVAL
    assert lib.bssn_rk4_plan_set_tile(None, 0, 6) == EINVAL
    assert lib.bssn_rk4_plan_destroy(None) == EINVAL
    count = C.c_int()
    assert lib.bssn_rk4_plan_violations(None, C.byref(count)) == EINVAL


def test_elementwise_arguments():
    assert lib.bssn_rk4_stage_f64(4, PTRS, PTRS, PTRS, C.c_int64(10), C.c_double(0.1), 1,
                                  C.c_double(1e-4), None, None) == EINVAL
    assert lib.bssn_rk4_stage_f64(0, PTRS, PTRS, PTRS, C.c_int64(-1), C.c_double(0.1), 1,
                                  C.c_double(1e-4), None, None) == EINVAL
    assert lib.bssn_enforce_f64(PTRS, C.c_int64(-1), C.c_double(1e-4), None, None) == EINVAL
    # halo buffers: negative sizes rejected, empty exchanges are no-ops
    assert lib.bssn_halo_pack_f64(FAKE, PTRS, FAKE, -1, None) == EINVAL
    assert lib.bssn_halo_unpack_f64(PTRS, FAKE, FAKE, -1, None) == EINVAL
    assert lib.bssn_halo_pack_f64(None, None, None, 0, None) == 0


def test_mesh_generator_and_partition_arguments():
    dims = (C.c_int32 * 3)(2, 2, 2)
    p = (C.c_double * 4)(0.7, 0.2, 0.08, 0.02)
    n = C.c_int()
    G = (C.c_int32 * 3)()
    h = C.c_double()
    assert lib.bssn_mesh_generate(5, dims, p, 0, -8.0, 16.0, None, C.byref(n), G, C.byref(h)) == EINVAL
    p0 = (C.c_double * 4)(0.7, 0.0, 0.28, 0.02)
    assert lib.bssn_mesh_generate(1, dims, p0, 0, -8.0, 16.0, None, C.byref(n), G, C.byref(h)) == EINVAL
    spec = B.generate_mesh(0, (2, 2, 2))
    part = (C.c_int32 * spec.nblocks)()
    assert lib.bssn_mesh_partition(spec.blocks, spec.nblocks, 0, part) == EINVAL
    assert lib.bssn_mesh_partition(spec.blocks, 0, 2, part) == EINVAL


def test_remesh_arguments():
    lib.bssn_remesh_mlp_bwd_noalloc_bf16.argtypes = [C.c_void_p] * 5 + [C.c_int] + [C.c_void_p] * 3
    f = lib.bssn_remesh_mlp_bwd_noalloc_bf16
    assert f(FAKE, FAKE, FAKE, FAKE, FAKE, 16385, FAKE, FAKE, None) == ELIMIT
    assert f(FAKE, FAKE, FAKE, FAKE, FAKE, 0, FAKE, FAKE, None) == EINVAL
    assert f(None, FAKE, FAKE, FAKE, FAKE, 16, FAKE, FAKE, None) == EINVAL
    # exact test: variable count outside 1..24, tolerance not positive, no mesh
    w = lib.bssn_remesh_wavelet_f64
    assert w(FAKE, PTRS, 25, 1e-6, FAKE, None, None, None) == EINVAL
    assert w(FAKE, PTRS, 0, 1e-6, FAKE, None, None, None) == EINVAL
    assert w(FAKE, PTRS, 24, 0.0, FAKE, None, None, None) == EINVAL
    assert w(None, PTRS, 24, 1e-6, FAKE, None, None, None) == EINVAL
    assert lib.bssn_remesh_features_f64(None, PTRS, FAKE, None) == EINVAL
    # two-flag decision: thresholds out of order, audit fraction or keep factor
    # outside [0, 1], tolerance not positive, missing outputs
    d = lib.bssn_remesh_decide2_f64

    def dec(lo_r=0.1, hi_r=0.9, lo_k=0.1, hi_k=0.9, audit=0.05, tol=1e-6, kf=0.1, out=FAKE):
        return d(FAKE, PTRS, FAKE, FAKE, lo_r, hi_r, FAKE, FAKE, lo_k, hi_k, audit, 7, tol, kf,
                 out, FAKE, FAKE, FAKE, 1 << 30, None)
    assert dec(lo_r=0.9, hi_r=0.1) == EINVAL
    assert dec(lo_k=0.9, hi_k=0.1) == EINVAL
    assert dec(audit=1.5) == EINVAL
    assert dec(audit=-0.1) == EINVAL
    assert dec(kf=1.5) == EINVAL
    assert dec(kf=0.0) == EINVAL
    assert dec(tol=0.0) == EINVAL
    assert dec(out=None) == EINVAL


def test_tile_queries():
    assert lib.bssn_tile_mode(lib.bssn_tile_count()) == -1
    info = (C.c_int * 4)()
    assert lib.bssn_tile_info(-1, info) == EINVAL
    lib.bssn_tile_selfcheck.restype = C.c_long
    assert lib.bssn_tile_selfcheck(99) == -1
    modes = [lib.bssn_tile_mode(t) for t in range(lib.bssn_tile_count())]
    assert set(modes) == {0, 1, 2}  # fused, split, on chip
