"""Checkpoint / restart (csrc/checkpoint.cu, bssn_b200/checkpoint.py) against
the reference's BSSNCtx::write_checkpt / restore_checkpt
(BSSN_GR/src/bssnCtx.cpp:783-1170): slot rule, header keys, newest-slot
choice, byte-exact round trip of mesh and state, and the failure statuses.
Host arrays only (no GPU); the evolution restart is in test_gpu_checkpoint.py."""
import ctypes as C
import json
import os
import sys

import numpy as np
import pytest

sys.path.insert(0, os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "dendro-gr_b200"))

B = pytest.importorskip("bssn_b200")
from bssn_b200 import checkpoint as ck  # noqa: E402

# the keys BSSNCtx::write_checkpt puts in its .cp file (bssnCtx.cpp:829-857)
REFERENCE_KEYS = {
    "DENDRO_TS_TIME_BEGIN", "DENDRO_TS_TIME_END", "DENDRO_TS_ELEMENT_ORDER", "DENDRO_TS_TIME_CURRENT",
    "DENDRO_TS_STEP_CURRENT", "DENDRO_TS_TIME_STEP_SIZE", "DENDRO_TS_LAST_IO_TIME",
    "DENDRO_TS_WAVELET_TOLERANCE", "DENDRO_TS_LOAD_IMB_TOLERANCE", "DENDRO_TS_NUM_VARS",
    "DENDRO_TS_ACTIVE_COMM_SZ", "DENDRO_BH1_X", "DENDRO_BH1_Y", "DENDRO_BH1_Z", "DENDRO_BH2_X",
    "DENDRO_BH2_Y", "DENDRO_BH2_Z",
}


@pytest.fixture
def mesh_state():
    spec = B.generate_mesh(1, (1, 1, 1), seed=3)
    rng = np.random.default_rng(11)
    U = rng.standard_normal((24, spec.n_nodes))
    return spec, U


def test_slot_rule():
    # bssnCtx.cpp:786-789: slot 0 when step % (2 freq) == 0, else 1
    flag = C.c_int(0)
    idx = [B.lib.bssn_checkpoint_index(s, 5, 0, C.byref(flag)) for s in (0, 5, 10, 15, 20, 7)]
    assert idx == [0, 1, 0, 1, 0, 1]
    # bssnCtx.cpp:791-796: the first checkpoint after the merger goes to slot 3, once
    assert B.lib.bssn_checkpoint_index(10, 5, 1, C.byref(flag)) == 3 and flag.value == 1
    assert B.lib.bssn_checkpoint_index(10, 5, 1, C.byref(flag)) == 0
    assert B.lib.bssn_checkpoint_index(10, 0, 0, C.byref(flag)) == -1


def test_round_trip_host(tmp_path, mesh_state):
    spec, U = mesh_state
    prefix = str(tmp_path / "bssn_cp")
    idx = ck.write_checkpoint(prefix, spec, U, step=10, time=2.5, dt=0.25, freq=5, time_end=100.0,
                              bh=((1.5, 0.25, 0.0), (-1.5, -0.25, 0.0)))
    assert idx == 0
    found = ck.latest_checkpoint(prefix)
    assert found is not None
    i, info = found
    assert i == 0 and info.step == 10 and info.time_current == 2.5 and info.time_step == 0.25
    assert info.time_end == 100.0 and info.num_vars == 24 and info.element_order == 6
    assert tuple(info.bh[0]) == (1.5, 0.25, 0.0) and tuple(info.bh[1]) == (-1.5, -0.25, 0.0)
    # header: a JSON object with exactly the reference's keys
    with open(prefix + "_step_0.cp") as f:
        hdr = json.load(f)
    assert set(hdr) == REFERENCE_KEYS
    assert hdr["DENDRO_TS_STEP_CURRENT"] == 10 and hdr["DENDRO_TS_LAST_IO_TIME"] == 2.5
    # mesh: identical descriptors and grid
    spec2 = ck.read_checkpoint_mesh(prefix, 0)
    assert spec2.nblocks == spec.nblocks and spec2.G == spec.G and spec2.h == spec.h
    assert spec2.origin3 == spec.origin3
    assert bytes(spec2.blocks) == bytes(spec.blocks)
    # state: bit-identical
    V = np.zeros_like(U)
    ck.read_checkpoint_vars(prefix, 0, V)
    assert np.array_equal(V.view(np.uint64), U.view(np.uint64))


def test_newest_slot_wins(tmp_path, mesh_state):
    spec, U = mesh_state
    prefix = str(tmp_path / "cp")
    assert ck.latest_checkpoint(prefix) is None
    assert ck.write_checkpoint(prefix, spec, U, step=10, time=1.0, dt=0.1, freq=5) == 0
    assert ck.write_checkpoint(prefix, spec, U + 1.0, step=15, time=1.5, dt=0.1, freq=5) == 1
    i, info = ck.latest_checkpoint(prefix)
    assert (i, info.step) == (1, 15)
    V = np.zeros_like(U)
    ck.read_checkpoint_vars(prefix, i, V)
    assert np.array_equal(V, U + 1.0)
    assert ck.write_checkpoint(prefix, spec, U + 2.0, step=20, time=2.0, dt=0.1, freq=5) == 0
    i, info = ck.latest_checkpoint(prefix)
    assert (i, info.step) == (0, 20)


def test_failures(tmp_path, mesh_state):
    spec, U = mesh_state
    prefix = str(tmp_path / "cp")
    ck.write_checkpoint(prefix, spec, U, step=0, time=0.0, dt=0.1)
    V = np.zeros_like(U)
    # wrong size
    with pytest.raises(B.BssnError):
        ck.read_checkpoint_vars(prefix, 0, np.zeros((24, spec.n_nodes - 1)))
    # a flipped byte in the variables fails the checksum
    var = prefix + "_0_0.var"
    raw = bytearray(open(var, "rb").read())
    raw[len(raw) // 2] ^= 0x10
    open(var, "wb").write(bytes(raw))
    n = (C.c_void_p * 24)(*[V.ctypes.data + v * V.shape[1] * 8 for v in range(24)])
    assert B.lib.bssn_checkpoint_read_vars(prefix.encode(), 0, 0, n, V.shape[1], None) == ck.EIO
    # a flipped byte in the block list fails the checksum
    oct_ = prefix + "_octree_0_0.oct"
    raw = bytearray(open(oct_, "rb").read())
    raw[100] ^= 0x01
    open(oct_, "wb").write(bytes(raw))
    with pytest.raises(B.BssnError):
        ck.read_checkpoint_mesh(prefix, 0)
    # a header that does not parse
    open(prefix + "_step_0.cp", "w").write('{"DENDRO_TS_STEP_CURRENT": \n')
    idx, info = C.c_int(), ck.CheckpointInfo()
    assert B.lib.bssn_checkpoint_latest(prefix.encode(), C.byref(idx), C.byref(info)) == ck.EIO
    # missing files
    assert B.lib.bssn_checkpoint_read_vars(str(tmp_path / "none").encode(), 0, 0, n, V.shape[1],
                                           None) == ck.ENOENT
    with pytest.raises(FileNotFoundError):
        ck.restore_checkpoint(str(tmp_path / "none"), device="cpu")
    # no temporary files left behind
    assert not [f for f in os.listdir(tmp_path) if f.endswith(".tmp")]
