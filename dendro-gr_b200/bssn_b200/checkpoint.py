"""Checkpoint and restart of an evolution: the reference's
BSSNCtx::write_checkpt / restore_checkpt (BSSN_GR/src/bssnCtx.cpp:783-1170)
over this library's mesh and zipped state (native code in
csrc/checkpoint.cu).

    idx = write_checkpoint(prefix, spec, U, step=s, time=t, dt=dt)
    spec, U, info = restore_checkpoint(prefix)          # newest of slots 0 / 1

Files: <prefix>_step_<i>.cp (JSON, the reference's keys, written by rank 0),
<prefix>_octree_<i>_<r>.oct (rank r's mesh) and <prefix>_<i>_<r>.var (rank
r's 24 zipped variables).  Slot i alternates with the step as the
reference's does: 0 when step % (2 * freq) == 0, else 1; 3 for the first
checkpoint after the punctures merged (distance below 0.1).
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import NVARS, BssnBlockDesc, MeshSpec, check, lib, stream_ptr

EIO = 7
ENOENT = 8


class CheckpointInfo(C.Structure):
    """BssnCheckpointInfo (include/bssn_b200.h): the .cp header."""
    _fields_ = [("time_begin", C.c_double), ("time_end", C.c_double),
                ("time_current", C.c_double), ("time_step", C.c_double),
                ("step", C.c_int64), ("element_order", C.c_int32), ("num_vars", C.c_int32),
                ("active_comm_size", C.c_int32), ("reserved", C.c_int32),
                ("wavelet_tol", C.c_double), ("load_imb_tol", C.c_double),
                ("bh", (C.c_double * 3) * 2)]


_P = C.c_void_p
lib.bssn_checkpoint_index.argtypes = [C.c_int64, C.c_int, C.c_int, C.POINTER(C.c_int)]
lib.bssn_checkpoint_write.argtypes = [C.c_char_p, C.c_int, C.c_int, C.c_int, C.POINTER(CheckpointInfo),
                                      C.POINTER(BssnBlockDesc), C.c_int, C.POINTER(C.c_int32),
                                      C.c_double, C.POINTER(C.c_double), _P, C.c_int64, _P]
lib.bssn_checkpoint_latest.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(CheckpointInfo)]
lib.bssn_checkpoint_read_mesh.argtypes = [C.c_char_p, C.c_int, C.c_int, C.POINTER(BssnBlockDesc),
                                          C.POINTER(C.c_int), C.POINTER(C.c_int32), C.POINTER(C.c_double),
                                          C.POINTER(C.c_double)]
lib.bssn_checkpoint_read_vars.argtypes = [C.c_char_p, C.c_int, C.c_int, _P, C.c_int64, _P]


class _MergeState:
    """The reference's BSSN_MERGED_CHKPT_WRITTEN flag, one per process."""
    written = C.c_int(0)


def checkpoint_index(step, freq, merged=False):
    """Slot of a checkpoint at `step` (bssnCtx.cpp:786-796)."""
    return lib.bssn_checkpoint_index(int(step), int(freq), int(bool(merged)), C.byref(_MergeState.written))


def _row_ptrs(U, stream=None):
    """24 pointers to the rows of a (24, n) float64 tensor or array (device
    or host memory), n, and the stream for the copies (none for host
    memory)."""
    try:
        import torch
        if isinstance(U, torch.Tensor):
            assert U.dtype == torch.float64 and U.is_contiguous() and U.shape[0] == NVARS
            n = U.shape[1]
            s = stream_ptr(stream) if U.is_cuda else C.c_void_p(0)
            return (C.c_void_p * NVARS)(*[U.data_ptr() + v * n * 8 for v in range(NVARS)]), n, s
    except ImportError:
        pass
    assert isinstance(U, np.ndarray) and U.dtype == np.float64 and U.flags.c_contiguous and U.shape[0] == NVARS
    n = U.shape[1]
    return (C.c_void_p * NVARS)(*[U.ctypes.data + v * n * 8 for v in range(NVARS)]), n, C.c_void_p(0)


def write_checkpoint(prefix, spec: MeshSpec, U, *, step, time, dt, freq=1, index=None, rank=0,
                     write_header=None, time_begin=0.0, time_end=0.0, element_order=6,
                     wavelet_tol=1e-6, load_imb_tol=0.1, active_comm_size=1,
                     bh=((1.0, 0.0, 0.0), (-1.0, 0.0, 0.0)), stream=None):
    """Write rank `rank`'s mesh and state U ((24, n_nodes) float64, CUDA
    tensor or host array) to slot `index` (default: the reference's slot rule
    with checkpoint frequency `freq`), and the JSON header on rank 0.
    Returns the slot."""
    if index is None:
        merged = float(np.linalg.norm(np.subtract(bh[0], bh[1]))) < 0.1
        index = checkpoint_index(step, freq, merged)
    if write_header is None:
        write_header = rank == 0
    info = CheckpointInfo()
    info.time_begin, info.time_end, info.time_current, info.time_step = time_begin, time_end, time, dt
    info.step, info.element_order, info.num_vars = int(step), element_order, NVARS
    info.active_comm_size, info.wavelet_tol, info.load_imb_tol = active_comm_size, wavelet_tol, load_imb_tol
    for i in range(2):
        for d in range(3):
            info.bh[i][d] = float(bh[i][d])
    ptr, n, sp = _row_ptrs(U, stream)
    assert n == spec.n_nodes, "state does not match the mesh"
    G = (C.c_int32 * 3)(*spec.G)
    org = (C.c_double * 3)(*spec.origin3)
    check(lib.bssn_checkpoint_write(prefix.encode(), index, rank, int(bool(write_header)), C.byref(info),
                                    spec.blocks, spec.nblocks, G, spec.h, org, ptr, n, sp),
          "checkpoint_write")
    return index


def latest_checkpoint(prefix):
    """(slot, CheckpointInfo) of the newest of slots 0 and 1, or None when
    neither header exists (bssnCtx.cpp:893-951)."""
    idx = C.c_int(-1)
    info = CheckpointInfo()
    rc = lib.bssn_checkpoint_latest(prefix.encode(), C.byref(idx), C.byref(info))
    if rc == ENOENT:
        return None
    check(rc, "checkpoint_latest")
    return idx.value, info


def read_checkpoint_mesh(prefix, index, rank=0) -> MeshSpec:
    n = C.c_int(0)
    G = (C.c_int32 * 3)()
    h = C.c_double(0)
    org = (C.c_double * 3)()
    check(lib.bssn_checkpoint_read_mesh(prefix.encode(), index, rank, None, C.byref(n), G, C.byref(h), org),
          "checkpoint_read_mesh")
    blocks = (BssnBlockDesc * n.value)()
    check(lib.bssn_checkpoint_read_mesh(prefix.encode(), index, rank, blocks, C.byref(n), G, C.byref(h), org),
          "checkpoint_read_mesh")
    sides = np.array([blocks[b].sz for b in range(n.value)], dtype=np.int32)
    origin = tuple(org)
    iso = origin[0] == origin[1] == origin[2]
    return MeshSpec(blocks, n.value, tuple(G), h.value, origin[0], sides, None if iso else origin)


def read_checkpoint_vars(prefix, index, U, rank=0, stream=None):
    """Fill U ((24, n_nodes) float64, CUDA tensor or host array) from rank
    `rank`'s .var file of slot `index`."""
    ptr, n, sp = _row_ptrs(U, stream)
    check(lib.bssn_checkpoint_read_vars(prefix.encode(), index, rank, ptr, n, sp),
          "checkpoint_read_vars")


def restore_checkpoint(prefix, rank=0, device="cuda"):
    """(spec, U, info) from the newest checkpoint: the rank's mesh, its state
    as a (24, n_nodes) float64 tensor on `device`, and the header.  Raises
    FileNotFoundError when no checkpoint exists."""
    import torch
    found = latest_checkpoint(prefix)
    if found is None:
        raise FileNotFoundError(f"no checkpoint {prefix}_step_{{0,1}}.cp")
    index, info = found
    spec = read_checkpoint_mesh(prefix, index, rank)
    U = torch.empty((NVARS, spec.n_nodes), dtype=torch.float64, device=device)
    read_checkpoint_vars(prefix, index, U, rank)
    if U.is_cuda:
        torch.cuda.synchronize()
    return spec, U, info
