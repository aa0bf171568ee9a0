"""Oracle of the multi-level mesh (test infrastructure): the level rules of
include/bssn_b200.h (BssnLevelBox) restated geometrically in numpy, with no
use of the library's maps, so the library's host-built maps and its GPU
kernels can be checked against it.

The reference takes its level transitions from dendrolib's ot::Mesh, which
is absent from the reference tree (call sites BSSN_GR/src/rkBSSN.cpp:611-650),
so these rules are this library's own definition (parity unpinned): the
interpolation is dendrolib's kind -- the parent element's degree-6 Lagrange
polynomial on its 7 nodes per axis -- evaluated axis by axis, x then y then
z, each product and sum rounded in that order (exactly what the GPU does).
The right-hand side per block and the enforcement are the reference's own
arithmetic through the compiled oracle (oracle_lib)."""
import ctypes as C

import numpy as np

from oracle_lib import NVARS, MeshOracle, rows

OCT = 6
RK4_C = (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0)
RK4_U = (0.0, 1.0 / 2.0, 1.0 / 2.0, 1.0)


def lagrange_half():
    """W[j][m]: degree-6 Lagrange weight of node m (0..6) at x = j + 1/2."""
    W = np.zeros((6, 7))
    for j in range(6):
        for m in range(7):
            num, den = 1, 1
            for k in range(7):
                if k != m:
                    num *= 2 * j + 1 - 2 * k
                    den *= 2 * (m - k)
            W[j, m] = num / den  # exact integers, one correctly rounded division
    return W


class LevelOracle:
    """Per patch (one per level for a box-per-level spec): its box, grid
    offset, parent and children, derived from the spec's patch list; every
    rule evaluated geometrically."""

    def __init__(self, spec, O):
        self.spec, self.O = spec, O
        self.W = lagrange_half()
        pl = spec.patch_list
        self.level = [int(p[0]) for p in pl]
        self.parent = [int(p[1]) for p in pl]
        self.boxes = [(np.array(p[2], dtype=np.int64), np.array(p[3], dtype=np.int64)) for p in pl]
        self.L = len(self.boxes)            # number of patches
        self.kids = [[c for c in range(self.L) if self.parent[c] == q] for q in range(self.L)]
        self.offsets, self.dims = [], []
        off = 0
        for lo, n in self.boxes:
            d = OCT * n + 1
            self.offsets.append(off)
            self.dims.append(d)
            off += int(np.prod(d))
        self.n_nodes = off
        bl = spec.as_numpy()
        self.blk = bl
        # the patch of every block: its level's patch holding its octants
        self.patch = np.full(spec.nblocks, -1, dtype=np.int64)
        self.octs = []
        for q, (lo, n) in enumerate(self.boxes):
            t = -np.ones(tuple(n[::-1]), dtype=np.int64)
            for b in np.nonzero(bl["level"] == self.level[q])[0]:
                o = bl["g0"][b] // OCT - lo
                w = (int(bl["sz"][b]) - 7) // OCT
                if np.all(o >= 0) and np.all(o + w <= n):
                    t[o[2]:o[2] + w, o[1]:o[1] + w, o[0]:o[0] + w] = b
                    self.patch[b] = q
            self.octs.append(t)
        assert (self.patch >= 0).all()
        self.mo = MeshOracle(spec, O)

    # ---- geometry
    def in_grid(self, l, q):
        lo, n = self.boxes[l]
        return np.all((q >= OCT * lo) & (q <= OCT * (lo + n)), axis=-1)

    def node(self, l, q):
        lo, _ = self.boxes[l]
        r = q - OCT * lo
        d = self.dims[l]
        return self.offsets[l] + r[..., 0] + d[0] * (r[..., 1] + d[1] * r[..., 2])

    def coarse_values(self, Z, l, q):
        """(24, N) values at patch-l points q (N, 3) from its parent: the
        coincident node, or the interpolation along every odd axis."""
        pa = self.parent[l]
        out = np.zeros((NVARS, len(q)))
        odd = (q & 1) == 1
        c = np.where(odd, OCT * (((q - 1) // 2) // OCT), q // 2)
        j = np.where(odd, (q - 1) // 2 - c, -1)
        pattern = odd[:, 0] * 1 + odd[:, 1] * 2 + odd[:, 2] * 4
        for pat in np.unique(pattern):
            sel = np.nonzero(pattern == pat)[0]
            cs, js = c[sel], j[sel]
            n = [7 if (pat >> d) & 1 else 1 for d in range(3)]
            wt = [self.W[np.maximum(js[:, d], 0)] if n[d] == 7 else np.ones((len(sel), 1)) for d in range(3)]
            tz = None
            for cc in range(n[2]):
                ty = None
                for bb in range(n[1]):
                    tx = None
                    for aa in range(n[0]):
                        p = cs + np.array([aa, bb, cc])
                        v = Z[:, self.node(pa, p)]
                        t = wt[0][:, aa] * v
                        tx = t if aa == 0 else tx + t
                    t = wt[1][:, bb] * tx
                    ty = t if bb == 0 else ty + t
                t = wt[2][:, cc] * ty
                tz = t if cc == 0 else tz + t
            out[:, sel] = tz
        return out

    # ---- ghost fill / owners / sync
    def unzip(self, Z):
        P = np.zeros((NVARS, self.spec.n_unzip))
        for b in range(self.spec.nblocks):
            s, l = int(self.blk["sz"][b]), int(self.patch[b])
            i = np.arange(s)
            qz, qy, qx = np.meshgrid(i, i, i, indexing="ij")
            q = np.stack([qx.ravel(), qy.ravel(), qz.ravel()], axis=1) + self.blk["g0"][b] - 3
            vals = np.zeros((NVARS, len(q)))
            ins = self.in_grid(l, q)
            vals[:, ins] = Z[:, self.node(l, q[ins])]
            if self.level[l] > 0 and (~ins).any():
                vals[:, ~ins] = self.coarse_values(Z, l, q[~ins])
            off = int(self.blk["offset"][b])
            P[:, off:off + s ** 3] = vals
        return P

    def owners(self):
        """Per node: the padded index of the zone that owns it, -1 if none."""
        own = -np.ones(self.n_nodes, dtype=np.int64)
        for l, (lo, n) in enumerate(self.boxes):
            d = self.dims[l]
            z, y, x = np.meshgrid(*[np.arange(k) for k in d[::-1]], indexing="ij")
            e = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
            q = e + OCT * lo
            keep = np.ones(len(q), dtype=bool)
            if self.level[l] > 0:
                keep &= ~np.any((e == 0) | (e == d - 1), axis=1)
            for c in self.kids[l]:
                clo, cn = self.boxes[c][0] // 2, self.boxes[c][1] // 2
                keep &= ~np.all((q > OCT * clo) & (q < OCT * (clo + cn)), axis=1)
            q = q[keep]
            t = np.minimum(q // OCT, lo + n - 1)
            b = self.octs[l][t[:, 2] - lo[2], t[:, 1] - lo[1], t[:, 0] - lo[0]]
            for c in self.kids[l]:  # on a finer patch's boundary: the octant below
                clo, cn = self.boxes[c][0] // 2, self.boxes[c][1] // 2
                m = (b < 0) & np.all((t >= clo) & (t < clo + cn), axis=1)
                if m.any():
                    t2 = t[m] - (q[m] == OCT * clo)
                    b[m] = self.octs[l][t2[:, 2] - lo[2], t2[:, 1] - lo[1], t2[:, 0] - lo[0]]
            assert (b >= 0).all()
            sz = self.blk["sz"][b].astype(np.int64)
            loc = q - self.blk["g0"][b] + 3
            own[self.node(l, q)] = self.blk["offset"][b] + loc[:, 0] + sz * (loc[:, 1] + sz * loc[:, 2])
        return own

    def sync(self, Z):
        order = sorted(range(1, self.L), key=lambda q: -self.level[q])
        for l in order:  # restriction, finest first
            lo, n = self.boxes[l]
            r = [np.arange(3 * lo[k] + 1, 3 * (lo[k] + n[k])) for k in range(3)]
            z, y, x = np.meshgrid(r[2], r[1], r[0], indexing="ij")
            c = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
            Z[:, self.node(self.parent[l], c)] = Z[:, self.node(l, 2 * c)]
        for l in sorted(range(1, self.L), key=lambda q: self.level[q]):  # boundaries, coarsest first
            lo, n = self.boxes[l]
            d = self.dims[l]
            z, y, x = np.meshgrid(*[np.arange(k) for k in d[::-1]], indexing="ij")
            e = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1)
            e = e[np.any((e == 0) | (e == d - 1), axis=1)]
            q = e + OCT * lo
            Z[:, self.node(l, q)] = self.coarse_values(Z, l, q)
        return Z

    # ---- evolution
    def initial_data(self, bh=(1.0, 0.0, 0.0, -1.0, 0.0, 0.0), m1=0.5, m2=0.5, chi_floor=1e-4, eps=1e-8,
                     seed=20261203):
        Z = np.zeros((NVARS, self.n_nodes))
        b = (C.c_double * 6)(*bh)
        for l, (lo, n) in enumerate(self.boxes):
            h = self.spec.h0 / 2 ** self.level[l]
            G = (C.c_int32 * 3)(*[int(x) for x in self.dims[l]])
            xm = (C.c_double * 3)(*[self.spec.xmin + OCT * int(lo[k]) * h for k in range(3)])
            ptr = (C.c_void_p * NVARS)(*[Z.ctypes.data + (v * self.n_nodes + self.offsets[l]) * 8
                                         for v in range(NVARS)])
            self.O.lib.orc_initial_data(ptr, G, xm, C.c_double(h), b, C.c_double(m1), C.c_double(m2),
                                        C.c_double(chi_floor), C.c_double(eps), C.c_uint64(seed + l))
        return self.sync(Z)

    def rk4_step(self, Z, dt, prm, chi_floor=1e-4):
        """One RK4 step with enforcement of every stage state, the GPU plan's
        order: ghost fill, right-hand side per block, owner gather (0 where
        no block owns), stage algebra, enforcement, level sync."""
        own = self.owners()
        u = Z.copy()
        acc = None
        im = Z
        for stage in range(4):
            R = self.mo.rhs(self.unzip(im if stage else u), prm)
            k = np.zeros((NVARS, self.n_nodes))
            m = own >= 0
            k[:, m] = R[:, own[m]]
            cc = RK4_C[stage] * dt
            if stage < 3:
                cu = RK4_U[stage + 1] * dt
                acc = (u if stage == 0 else acc) + cc * k
                im = np.ascontiguousarray(u + cu * k)
                self.O.lib.orc_enforce(rows(im), C.c_int64(self.n_nodes), C.c_double(chi_floor))
                im = self.sync(im)
            else:
                out = np.ascontiguousarray(acc + cc * k)
                self.O.lib.orc_enforce(rows(out), C.c_int64(self.n_nodes), C.c_double(chi_floor))
                return self.sync(out)


def transfer(LO_old, Z_old, LO_new):
    """State on LO_new's hierarchy from Z_old on LO_old's: per new patch,
    parents first, the node of an old patch of the same level where one has
    it, else the coincident node or interpolation from the new parent; then
    the new hierarchy's sync."""
    Z = np.zeros((NVARS, LO_new.n_nodes))
    for l, (lo, n) in enumerate(LO_new.boxes):
        d = LO_new.dims[l]
        z, y, x = np.meshgrid(*[np.arange(k) for k in d[::-1]], indexing="ij")
        q = np.stack([x.ravel(), y.ravel(), z.ravel()], axis=1) + OCT * lo
        done = np.zeros(len(q), dtype=bool)
        for r in range(LO_old.L):  # the old patch of the same level holding the node
            if LO_old.level[r] != LO_new.level[l]:
                continue
            m = ~done & LO_old.in_grid(r, q)
            if m.any():
                Z[:, LO_new.node(l, q[m])] = Z_old[:, LO_old.node(r, q[m])]
                done |= m
        if (~done).any():
            assert LO_new.level[l] > 0
            Z[:, LO_new.node(l, q[~done])] = LO_new.coarse_values(Z, l, q[~done])
    return LO_new.sync(Z)
