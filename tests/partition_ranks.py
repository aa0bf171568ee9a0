"""Rank bodies of the partitioned-evolution tests (run in spawned processes).

Each rank builds its box mesh and halo lists from the global mesh, takes its
box of the global initial state, advances it by RK4 steps with the halo
exchange before every stage, and saves the values of the nodes it owns.
The CPU body uses the oracle as the engine (unzip, right-hand side, zip and
the stage algebra of BSSN_GR/src/rkBSSN.cpp:764-860, as the oracle's own
orc_rk4_step does them); the GPU body uses the library's partitioned plan.
"""
import os
import sys
from datetime import timedelta

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "dendro-gr_b200"))

RK4_C = (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0)
RK4_U = (0.0, 1.0 / 2.0, 1.0 / 2.0, 1.0)


def mesh(kind):
    import bssn_b200 as B
    if kind == "uniform":
        return B.generate_mesh(0, (4, 4, 4))
    return B.generate_mesh(1, (2, 1, 1), seed=1, xmin=-8.25)


def box_global_ids(sub, G):
    """Global node index of every node of the rank's box."""
    L = sub.spec.G
    n = np.arange(sub.n_nodes, dtype=np.int64)
    x = n % L[0] + sub.lo[0]
    y = (n // L[0]) % L[1] + sub.lo[1]
    z = n // (L[0] * L[1]) + sub.lo[2]
    return x + G[0] * (y + G[1] * z)


def _init(rank, world, port, backend):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group(backend, rank=rank, world_size=world, timeout=timedelta(seconds=120))


def oracle_steps(Z, mo, ex, O, dt, steps):
    """RK4 steps of a rank's box state with the oracle, the halo nodes
    refreshed by the exchange before every stage."""
    import torch
    import oracle_lib as ol
    prm = ol.params()
    for _ in range(steps):
        ex.run(torch.from_numpy(Z))
        prev = Z.copy()
        ks = []
        im = np.zeros_like(Z)
        for stage in range(4):
            src = Z if stage == 0 else im
            if stage > 0:
                ex.run(torch.from_numpy(im))
            k = mo.zip(mo.rhs(mo.unzip(src), prm))
            ks.append(k)
            if stage < 3:
                im = prev + (RK4_U[stage + 1] * dt) * k
                O.lib.orc_enforce(ol.rows(im), C_int64(im.shape[1]), C_double(1e-4))
        Z = prev.copy()
        for s in range(4):
            Z += (RK4_C[s] * dt) * ks[s]
        O.lib.orc_enforce(ol.rows(Z), C_int64(Z.shape[1]), C_double(1e-4))
    return Z


def cpu_rank(rank, world, port, kind, steps, outdir):
    import torch
    import torch.distributed as dist
    import oracle_lib as ol
    from bssn_b200.distributed import HaloExchange, partition, subdomain
    _init(rank, world, port, "gloo")
    try:
        spec = mesh(kind)
        O = ol.oracle()
        Z0 = ol.MeshOracle(spec, O).initial_data(eps=1e-8)
        part = partition(spec, world)
        sub = subdomain(spec, part, rank)
        Z = np.ascontiguousarray(Z0[:, box_global_ids(sub, spec.G)])
        mo = ol.MeshOracle(sub.spec, O)
        ex = HaloExchange(sub, torch.device("cpu"))
        Z = oracle_steps(Z, mo, ex, O, 0.25 * spec.h, steps)
        np.save(os.path.join(outdir, f"vals{rank}.npy"), Z[:, sub.owned])
        np.save(os.path.join(outdir, f"ids{rank}.npy"), sub.owned_global)
    finally:
        dist.destroy_process_group()


def block_flags(spec, U, O, tol=1e-6):
    """Per-block exact wavelet flags of a ghost-filled state U (any element
    and variable above tol), from the oracle's scores."""
    import oracle_lib as ol
    ne = int(sum(((int(s) - 7) // 6) ** 3 for s in spec.sides))
    sc = np.zeros(ne * 24)
    O.lib.orc_wavelet_scores(ol.rows(U), spec.blocks, spec.nblocks, 24, sc.ctypes.data_as(ol._dp))
    first = np.cumsum([0] + [((int(s) - 7) // 6) ** 3 for s in spec.sides])
    sc = sc.reshape(ne, 24)
    return np.array([sc[first[b]:first[b + 1]].max() > tol for b in range(spec.nblocks)])


def owned_sums(sub, cons, bh=(1.0, 0.0, 0.0, -1.0, 0.0, 0.0), radii=(0.5, 0.5)):
    """Sums of squares of the 4 constraint fields and the node count over the
    nodes the rank owns outside both radii (coordinates on the rank's box)."""
    spec = sub.spec
    o, G, h = spec.origin3, spec.G, spec.h
    g = sub.owned
    x = o[0] + (g % G[0]) * h
    y = o[1] + ((g // G[0]) % G[1]) * h
    z = o[2] + (g // (G[0] * G[1])) * h
    d1 = np.sqrt((x - bh[0]) ** 2 + (y - bh[1]) ** 2 + (z - bh[2]) ** 2)
    d2 = np.sqrt((x - bh[3]) ** 2 + (y - bh[4]) ** 2 + (z - bh[5]) ** 2)
    sel = g[~((d1 < radii[0]) | (d2 < radii[1]))]
    return np.array([(cons[c, sel] ** 2).sum() for c in range(4)] + [float(len(sel))])


def cpu_diag_rank(rank, world, port, kind, steps, outdir):
    """After `steps` partitioned oracle steps: the constraint norms from the
    ranks' owned-node sums reduced over the ranks, the per-block wavelet
    flags of the rank's blocks, the remesh OR-vote and the time-step
    minimum."""
    import torch
    import torch.distributed as dist
    import oracle_lib as ol
    from bssn_b200.distributed import (HaloExchange, allreduce_sum, dt_min, norms_from_sums, partition,
                                       remesh_vote, subdomain)
    _init(rank, world, port, "gloo")
    try:
        spec = mesh(kind)
        O = ol.oracle()
        Z0 = ol.MeshOracle(spec, O).initial_data(eps=1e-8)
        part = partition(spec, world)
        sub = subdomain(spec, part, rank)
        Z = np.ascontiguousarray(Z0[:, box_global_ids(sub, spec.G)])
        mo = ol.MeshOracle(sub.spec, O)
        ex = HaloExchange(sub, torch.device("cpu"))
        dt = 0.25 * spec.h
        Z = oracle_steps(Z, mo, ex, O, dt, steps)
        ex.run(torch.from_numpy(Z))
        U = mo.unzip(Z)
        cons = ol.oracle_constraints(sub.spec, U, O)
        sums = allreduce_sum(torch.from_numpy(owned_sums(sub, cons)))
        np.save(os.path.join(outdir, f"norms{rank}.npy"), norms_from_sums(sums.numpy()))
        flags = block_flags(sub.spec, U, O)
        np.save(os.path.join(outdir, f"flags{rank}.npy"), np.stack([sub.blocks, flags.astype(np.int64)]))
        np.save(os.path.join(outdir, f"vote{rank}.npy"), np.array([remesh_vote(flags.any()),
                                                                    remesh_vote(rank == world - 1),
                                                                    remesh_vote(False)]))
        np.save(os.path.join(outdir, f"dt{rank}.npy"), np.array([dt_min(dt * (1 + rank))]))
    finally:
        dist.destroy_process_group()


def gpu_rank(rank, world, port, kind, steps, outdir):
    import torch
    import torch.distributed as dist
    import bssn_b200 as B
    import oracle_lib as ol
    from bssn_b200.distributed import PartitionedRK4
    _init(rank, world, port, "gloo")
    try:
        torch.cuda.set_device(0)
        spec = mesh(kind)
        Z0 = ol.MeshOracle(spec, ol.oracle()).initial_data(eps=1e-8)
        pr = PartitionedRK4(spec, rank, world)
        ids = box_global_ids(pr.sub, spec.G)
        U = torch.from_numpy(np.ascontiguousarray(Z0[:, ids])).cuda()
        for _ in range(steps):
            pr.step(U, 0.25 * spec.h)
        torch.cuda.synchronize()
        got = U.cpu().numpy()
        np.save(os.path.join(outdir, f"vals{rank}.npy"), got[:, pr.sub.owned])
        np.save(os.path.join(outdir, f"ids{rank}.npy"), pr.sub.owned_global)
        # the global constraint norms, reduced over the ranks (every rank calls it)
        np.save(os.path.join(outdir, f"norms{rank}.npy"), pr.constraint_norms(U))
        pr.close()
    finally:
        dist.destroy_process_group()


def C_double(v):
    import ctypes
    return ctypes.c_double(v)


def C_int64(v):
    import ctypes
    return ctypes.c_int64(v)
