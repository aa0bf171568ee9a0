"""Multi-GPU evolution: block partition with a halo exchange before every
RK4 stage (one process per GPU).

The blocks are split along their Z-order into ranges of about equal zone
counts (bssn_mesh_partition; the reference partitions its octree along a
space-filling curve).  Rank r evolves its own blocks as a mesh of their own
on the bounding box of the blocks' padded regions in the node grid, so the
library's ghost fill, right-hand side, owner rule and stage kernels run
unchanged on the box.  Every node of the box that r's blocks read but a block
of another rank owns (the zip's owner rule: a node on a block's upper face
belongs to the next block) is received from its owner before each stage, and
r sends the nodes it owns that other ranks read -- the reference's
ghostExchangeStart / ghostExchangeRecvSync around its unzip
(BSSN_GR/src/rkBSSN.cpp:620-641).  Lists are in increasing global node
order on both sides, so a send matches its receive element by element.

Transport: torch.distributed point-to-point (NCCL between GPUs; with the
gloo backend the buffers go through host memory).  The global quantities
are reductions over the ranks, as the reference's MPI reductions: the
constraint L2 norms from summed squares and counts of owned nodes, the time
step as a minimum, the remesh decision as a logical OR.  Packing and unpacking run
on the GPU (bssn_halo_pack_f64 / bssn_halo_unpack_f64), or, for host arrays,
as numpy gathers (the same lists).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import (NVARS, BssnBlockDesc, Mesh, MeshSpec, RK4Plan, PLAN_ENFORCE_STAGES, PLAN_GRAPH,
               check, default_params, lib, ptrs, stream_ptr)

lib.bssn_constraint_sums_f64.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_void_p, C.c_double,
                                         C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]

OCT = 6  # nodes per octant edge


def partition(spec: MeshSpec, nparts: int) -> np.ndarray:
    """Rank of every block (int32): nparts Z-order ranges, balanced by zones."""
    part = np.zeros(spec.nblocks, dtype=np.int32)
    check(lib.bssn_mesh_partition(spec.blocks, spec.nblocks, nparts,
                                  part.ctypes.data_as(C.POINTER(C.c_int32))), "mesh_partition")
    return part


def _padded_box(blk, G):
    """Inclusive node range [lo, hi] per axis read by a block's ghost fill:
    its padded region (3 nodes around the interior) clipped to the grid."""
    lo = np.array([max(int(blk.g0[d]) - 3, 0) for d in range(3)], dtype=np.int64)
    hi = np.array([min(int(blk.g0[d]) + int(blk.sz) - 4, int(G[d]) - 1) for d in range(3)], dtype=np.int64)
    return lo, hi


@dataclass
class Subdomain:
    """Rank `rank`'s part of a partitioned mesh."""
    spec: MeshSpec           # the rank's own mesh on its box
    lo: tuple                # global node of local node (0, 0, 0)
    blocks: np.ndarray       # global ids of the rank's blocks, in local order
    send: dict               # peer -> local node indices sent to it (int64)
    recv: dict               # peer -> local node indices received from it
    owned: np.ndarray        # local indices of the nodes this rank owns
    owned_global: np.ndarray  # their global node indices

    @property
    def n_nodes(self):
        return self.spec.n_nodes


def subdomain(spec: MeshSpec, part: np.ndarray, rank: int) -> Subdomain:
    """Build rank `rank`'s box mesh and halo lists (host, from the global
    block list; every rank computes its own lists).  All arrays span the
    rank's box only: every node the rank sends (owned by it) or receives
    (read by its blocks) lies in the box, and lexicographic (z, y, x) order
    is the same in the box and in the grid, so a send list (ordered on the
    sender's box) matches the receive list (ordered on the receiver's box)."""
    G = np.asarray(spec.G, dtype=np.int64)
    M = (G - 1) // OCT
    mine = np.nonzero(part == rank)[0]
    pads = [_padded_box(spec.blocks[b], G) for b in range(spec.nblocks)]
    # box: the union of the rank's padded boxes, widened to whole octants so
    # the box is a grid of its own (6M+1 nodes per axis, block origins on
    # octant corners)
    lo = np.min([pads[b][0] for b in mine], axis=0) // OCT * OCT
    hi = np.max([pads[b][1] for b in mine], axis=0)
    hi = np.minimum(lo + (hi - lo + OCT - 1) // OCT * OCT, G - 1)
    L = hi - lo + 1

    def touching(b):
        return bool((pads[b][0] <= hi).all() and (pads[b][1] >= lo).all())

    near = [b for b in range(spec.nblocks) if touching(b)]
    # owner rank of every box node: the rank of the block whose octants hold
    # the node's octant (the zip's owner rule); octant range of the box
    olo = lo // OCT
    ohi = np.minimum(hi // OCT, M - 1)
    omap = np.full(tuple((ohi - olo + 1)[::-1]), -1, dtype=np.int32)
    for b in near:
        blk = spec.blocks[b]
        o = np.array(blk.g0[:], dtype=np.int64) // OCT
        w = (int(blk.sz) - 7) // OCT
        a = np.maximum(o, olo) - olo
        e = np.minimum(o + w - 1, ohi) - olo + 1
        if (e > a).all():
            omap[a[2]:e[2], a[1]:e[1], a[0]:e[0]] = part[b]
    ax = [np.minimum((np.arange(L[d]) + lo[d]) // OCT, M[d] - 1) - olo[d] for d in range(3)]
    owner = omap[ax[2][:, None, None], ax[1][None, :, None], ax[0][None, None, :]].ravel()

    def mask_of(blocks):
        m = np.zeros((L[2], L[1], L[0]), dtype=bool)
        for b in blocks:
            a = np.maximum(pads[b][0], lo) - lo
            e = np.minimum(pads[b][1], hi) - lo + 1
            if (e > a).all():
                m[a[2]:e[2], a[1]:e[1], a[0]:e[0]] = True
        return m.ravel()

    needed = mask_of(mine)
    send, recv = {}, {}
    for q in sorted(set(int(part[b]) for b in near) - {rank}):
        r_ids = np.nonzero(needed & (owner == q))[0]
        s_ids = np.nonzero(mask_of([b for b in near if part[b] == q]) & (owner == rank))[0]
        if len(r_ids):
            recv[q] = r_ids.astype(np.int64)
        if len(s_ids):
            send[q] = s_ids.astype(np.int64)
    owned = np.nonzero(owner == rank)[0].astype(np.int64)
    ox = owned % L[0] + lo[0]
    oy = (owned // L[0]) % L[1] + lo[1]
    oz = owned // (L[0] * L[1]) + lo[2]
    # the rank's blocks, origins shifted into the box, offsets renumbered
    blocks = (BssnBlockDesc * len(mine))()
    off = 0
    for i, b in enumerate(mine):
        src = spec.blocks[int(b)]
        C.memmove(C.byref(blocks[i]), C.byref(src), C.sizeof(BssnBlockDesc))
        for d in range(3):
            blocks[i].g0[d] = int(src.g0[d]) - int(lo[d])
        blocks[i].offset = off
        n = int(src.sz) ** 3
        off += (n + 1) // 2 * 2
    origin = tuple(spec.origin3[d] + float(lo[d]) * spec.h for d in range(3))
    local = MeshSpec(blocks, len(mine), tuple(int(v) for v in L), spec.h, spec.xmin,
                     np.array([int(spec.blocks[int(b)].sz) for b in mine], dtype=np.int32), origin)
    return Subdomain(local, tuple(int(v) for v in lo), mine, send, recv, owned,
                     (ox + G[0] * (oy + G[1] * oz)).astype(np.int64))


class HaloExchange:
    """Per-stage exchange of a rank's halo nodes with torch.distributed
    point-to-point operations (every rank posts all its sends and receives
    in increasing peer order)."""

    def __init__(self, sub: Subdomain, device, group=None):
        import torch
        import torch.distributed as dist
        self.sub = sub
        self.device = device
        self.group = group
        self.peers = sorted(set(sub.send) | set(sub.recv))
        gpu = device.type == "cuda"
        # gloo moves host tensors only: device buffers then go through pinned
        # host copies
        self.via_host = bool(self.peers) and gpu and dist.get_backend(group) == "gloo"
        self.idx = {}
        self.sbuf, self.rbuf, self.hbuf = {}, {}, {}
        for q in self.peers:
            for kind, lists, bufs in (("s", sub.send, self.sbuf), ("r", sub.recv, self.rbuf)):
                if q in lists:
                    ix = torch.from_numpy(lists[q])
                    self.idx[(kind, q)] = ix.to(device) if gpu else ix
                    bufs[q] = torch.empty(NVARS * len(lists[q]), dtype=torch.float64, device=device)
                    if self.via_host:
                        self.hbuf[(kind, q)] = torch.empty(NVARS * len(lists[q]), dtype=torch.float64,
                                                           pin_memory=True)

    def run(self, fields):
        """fields: 24 device pointers (GPU) or a (24, n) float64 CPU tensor."""
        import torch
        import torch.distributed as dist
        gpu = self.device.type == "cuda"
        for q, buf in self.sbuf.items():
            ix = self.idx[("s", q)]
            if gpu:
                check(lib.bssn_halo_pack_f64(C.c_void_p(buf.data_ptr()), fields, C.c_void_p(ix.data_ptr()),
                                             len(ix), stream_ptr()), "halo_pack")
            else:
                buf.copy_(fields[:, ix].reshape(-1))
        send, recv = dict(self.sbuf), dict(self.rbuf)
        if self.via_host:
            for q in send:
                self.hbuf[("s", q)].copy_(send[q])
                send[q] = self.hbuf[("s", q)]
            for q in recv:
                recv[q] = self.hbuf[("r", q)]
        # NCCL orders its transfers after the packing on the current stream;
        # the gloo path's device-to-host copies above are synchronous
        ops = []
        for q in self.peers:
            if q in send:
                ops.append(dist.P2POp(dist.isend, send[q], q, group=self.group))
            if q in recv:
                ops.append(dist.P2POp(dist.irecv, recv[q], q, group=self.group))
        if ops:
            for req in dist.batch_isend_irecv(ops):
                req.wait()
        if self.via_host:
            for q in recv:
                self.rbuf[q].copy_(recv[q])
        for q, buf in self.rbuf.items():
            ix = self.idx[("r", q)]
            if gpu:
                check(lib.bssn_halo_unpack_f64(fields, C.c_void_p(buf.data_ptr()), C.c_void_p(ix.data_ptr()),
                                               len(ix), stream_ptr()), "halo_unpack")
            else:
                fields[:, ix] = buf.reshape(NVARS, -1)


# ---------------------------------------------------------------------------
# Reductions over the ranks (the reference's MPI reductions)
# ---------------------------------------------------------------------------
def allreduce_sum(t, group=None):
    """Sum a float64 tensor over the ranks, in place (NCCL for device
    tensors, gloo for host tensors)."""
    import torch.distributed as dist
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    return t


def norms_from_sums(sums):
    """Constraint L2 norms sqrt(sum c^2 / N) from the 5 reduced sums
    (bssn_constraint_sums_f64 layout: sums of squares, then the count)."""
    s = np.asarray(sums, dtype=np.float64)
    n = s[4]
    return np.sqrt(s[:4] / n) if n > 0 else np.zeros(4)


def dt_min(dt_local, group=None):
    """The global time step: the minimum of the ranks' CFL time steps (the
    reference reduces its dt with MPI_MIN, BSSN_GR/src/bssngr_main.cpp)."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(dt_local)], dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MIN, group=group)
    return float(t.item())


def remesh_vote(flag_local, group=None):
    """Whether any rank asks for a remesh: the reference's
    MPI_Allreduce(..., MPI_LOR) after isReMeshWAMR
    (BSSN_GR/src/dataUtils.cpp:833), as a MAX over 0/1."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([1 if flag_local else 0], dtype=torch.int32)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return bool(t.item())


def owned_mask(sub: Subdomain):
    """uint8 per node of the rank's box: 1 where the rank owns the node."""
    m = np.zeros(sub.n_nodes, dtype=np.uint8)
    m[sub.owned] = 1
    return m


class PartitionedRK4:
    """One rank's share of a partitioned RK4 evolution on its GPU: the
    rank's box mesh, an RK4 plan on it run stage by stage, and the halo
    exchange of the stage input before each stage."""

    def __init__(self, spec: MeshSpec, rank: int, world: int, params=None, group=None,
                 flags=PLAN_ENFORCE_STAGES, tile=None):
        import torch
        self.part = partition(spec, world)
        self.sub = subdomain(spec, self.part, rank)
        self.mesh = Mesh(self.sub.spec)
        # stages run one by one (eagerly) around the exchanges
        self.plan = RK4Plan(self.mesh, params or default_params(), flags & ~PLAN_GRAPH)
        if tile is not None:
            self.plan.set_tile(tile)
        im = (C.c_void_p * NVARS)()
        check(lib.bssn_rk4_plan_stage_state(self.plan.h, im), "stage_state")
        self.im = im
        self.ex = HaloExchange(self.sub, torch.device("cuda"), group)

    def step(self, U, dt):
        """Advance the rank's local state U ((24, n_local) CUDA tensor) by one
        RK4 step; the halo nodes are refreshed before every stage."""
        u = ptrs(U)
        for stage in range(4):
            self.ex.run(u if stage == 0 else self.im)
            check(lib.bssn_rk4_plan_stage(self.plan.h, u, dt, stage, stream_ptr()), "plan_stage")

    def constraint_norms(self, U, bh=(1.0, 0.0, 0.0, -1.0, 0.0, 0.0), radii=(0.5, 0.5)):
        """Hamiltonian / momentum constraint L2 norms of the whole
        partitioned state (every rank calls it): halo exchange of U, ghost
        fill and constraints on the rank's box, sums of squares over the
        nodes this rank owns outside the radii, summed over the ranks."""
        import torch
        from . import constraints
        if not hasattr(self, "_diag"):
            spec = self.sub.spec
            self._diag = (torch.zeros((NVARS, self.mesh.n_unzip), dtype=torch.float64, device="cuda"),
                          torch.zeros((4, spec.n_nodes), dtype=torch.float64, device="cuda"),
                          torch.from_numpy(owned_mask(self.sub)).cuda(),
                          torch.zeros(5, dtype=torch.float64, device="cuda"))
        Pz, cons, mask, sums = self._diag
        self.ex.run(ptrs(U))
        self.mesh.unzip(Pz, U)
        constraints(self.mesh, cons, Pz)
        spec = self.sub.spec
        cp = (C.c_void_p * 4)(*[cons[c].data_ptr() for c in range(4)])
        check(lib.bssn_constraint_sums_f64(self.mesh.h, cp, 4, (C.c_double * 3)(*spec.origin3), spec.h,
                                           (C.c_double * 6)(*bh), (C.c_double * 2)(*radii),
                                           C.c_void_p(mask.data_ptr()), C.c_void_p(sums.data_ptr()),
                                           stream_ptr()), "constraint_sums")
        allreduce_sum(sums, self.ex.group)
        return norms_from_sums(sums.cpu().numpy())

    def close(self):
        self.plan.close()
        self.mesh.close()
