"""Multi-rank evolution by block partition with a halo exchange before each
RK4 stage: two gloo ranks on the CPU, the oracle as the engine.
The partitioned step must reproduce the single-domain oracle step bit for
bit on every node, each node owned by exactly one rank."""
import os
import socket
import tempfile

import numpy as np
import pytest

import oracle_lib as ol
import partition_ranks as pr

torch = pytest.importorskip("torch")


def free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def run_ranks(fn, world, kind, steps, outdir):
    import torch.multiprocessing as mp
    ctx = mp.get_context("spawn")
    port = free_port()
    procs = [ctx.Process(target=fn, args=(r, world, port, kind, steps, outdir)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=600)
    for p in procs:
        if p.is_alive():
            p.kill()
        assert p.exitcode == 0, p.exitcode


def gather(outdir, world):
    ids = [np.load(os.path.join(outdir, f"ids{r}.npy")) for r in range(world)]
    vals = [np.load(os.path.join(outdir, f"vals{r}.npy")) for r in range(world)]
    return ids, vals


def reference_step(kind, steps):
    spec = pr.mesh(kind)
    mo = ol.MeshOracle(spec, ol.oracle())
    Z = mo.initial_data(eps=1e-8)
    for _ in range(steps):
        assert mo.rk4_step(Z, 0.25 * spec.h, ol.params()) == 0
    return spec, Z


def test_partition_balanced_and_contiguous():
    import bssn_b200 as B
    from bssn_b200.distributed import partition
    spec = B.generate_mesh(1, (4, 2, 2), seed=3)
    zones = (spec.sides.astype(np.int64) - 6) ** 3
    for n in (2, 3, 4, 8):
        part = partition(spec, n)
        assert set(part.tolist()) == set(range(n))
        share = np.array([zones[part == r].sum() for r in range(n)]) / zones.sum()
        assert share.max() < 1.0 / n + 0.05, share


@pytest.mark.parametrize("kind,world,steps", [("uniform", 2, 1), ("mix", 2, 1), ("mix", 3, 2)])
def test_partitioned_step_matches_single_domain(kind, world, steps):
    spec, Zref = reference_step(kind, steps)
    with tempfile.TemporaryDirectory() as d:
        run_ranks(pr.cpu_rank, world, kind, steps, d)
        ids, vals = gather(d, world)
    all_ids = np.concatenate(ids)
    assert len(all_ids) == spec.n_nodes and len(np.unique(all_ids)) == spec.n_nodes
    for i, v in zip(ids, vals):
        assert np.array_equal(v, Zref[:, i])


@pytest.mark.parametrize("kind,world", [("mix", 2), ("uniform", 3)])
def test_partitioned_reductions_match_single_domain(kind, world):
    """The global quantities of a partitioned run after one step: constraint
    L2 norms from the ranks' owned-node sums reduced over the ranks equal the
    single-domain norms; every block's exact wavelet flag equals its flag in
    the single domain; the remesh OR-vote and the time-step minimum are the
    same on every rank."""
    spec, Z = reference_step(kind, 1)
    O = ol.oracle()
    mo = ol.MeshOracle(spec, O)
    U = mo.unzip(Z)
    ref_norms = ol.l2_norms(spec, ol.oracle_constraints(spec, U, O))
    ref_flags = pr.block_flags(spec, U, O)
    with tempfile.TemporaryDirectory() as d:
        run_ranks(pr.cpu_diag_rank, world, kind, 1, d)
        norms = [np.load(os.path.join(d, f"norms{r}.npy")) for r in range(world)]
        flags = [np.load(os.path.join(d, f"flags{r}.npy")) for r in range(world)]
        votes = [np.load(os.path.join(d, f"vote{r}.npy")) for r in range(world)]
        dts = [np.load(os.path.join(d, f"dt{r}.npy"))[0] for r in range(world)]
    for n in norms:
        assert np.allclose(n, ref_norms, rtol=1e-12, atol=0), (n, ref_norms)
    got = np.full(spec.nblocks, -1)
    for f in flags:
        got[f[0]] = f[1]
    assert np.array_equal(got, ref_flags.astype(np.int64))
    for v in votes:
        assert list(v) == [bool(ref_flags.any()), True, False]
    assert dts == [0.25 * spec.h] * world
