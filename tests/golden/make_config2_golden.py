"""Regenerates tests/golden/config2_golden.npz: ten RK4 steps of the
mixed-size octree workload at the plain-path size -- 4,108 blocks of sides
13/19/31/55 drawn with block-count fractions 0.7/0.2/0.08/0.02 (the seeded
top-down split of 8 x 5 x 4 super-cells of 8^3 octants, the split closest
to 4,000 blocks; 19.76 M zones, spacing 1/12) on the box [-16, 16] x
[-10, 10] x [-8, 8] -- centred on the coordinate origin, from which the
Sommerfeld condition measures r, and reaching 8 from it on the shortest axis
as config 1's [-8, 8]^3 does -- shifted by half a cell (node (0,0,0) at
(-16, -10, -8) - 1/24) so that no node sits on a puncture,
Brill-Lindquist m1 = m2 = 0.5 at (+-1, 0, 0) plus a seeded 1e-8
perturbation, dt = 0.25 dx, KO sigma 0.4, eta 2 -- evolved on the CPU
with the reference's OWN compiled right-hand side (oracle/_ref, the block
loop of rhs.cpp over bssnrhs) inside the classical RK4 of
BSSN_GR/src/rkBSSN.cpp:764-860 with per-stage constraint enforcement (the
ghost fill, zip, stage algebra and enforcement restated in
oracle/bssn_oracle.cpp).  The mesh comes from the oracle's own generator,
so this script never loads the product library.

Stored (small enough to commit): per variable the largest magnitude and the
sum of squares over every node after step 10, the values of 4,096 seeded
nodes after step 10 (every variable), and the Hamiltonian / momentum
constraint L2 norms (outside r < 0.5 of each puncture) after every step.
Run from the repository root (about 10 minutes on 8 cores, 40 GB of RAM):

    python tests/golden/make_config2_golden.py
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import oracle_lib as ol  # noqa: E402

DIMS = (8, 5, 4)
SEED_MESH = 20261203
L = 32.0
ORIGIN = (-16.0 - 1.0 / 24.0, -10.0 - 1.0 / 24.0, -8.0 - 1.0 / 24.0)
STEPS = 10
NSAMPLE = 4096
RADII = (0.5, 0.5)
BH = (1.0, 0.0, 0.0, -1.0, 0.0, 0.0)


def sample_nodes(n_nodes):
    rng = np.random.default_rng(2026)
    return np.sort(rng.choice(n_nodes, NSAMPLE, replace=False)).astype(np.int64)


def main():
    ref = ol.reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libbssn_ref.so missing: run `make -C oracle REF=...`")
    O = ol.oracle()
    spec = ol.OracleMeshSpec(1, DIMS, seed=SEED_MESH, L=L, origin=ORIGIN)
    mo = ol.MeshOracle(spec, O)
    prm = ol.params()
    dt = 0.25 * spec.h
    Z = mo.initial_data(bh=BH, eps=1e-8)
    ws = mo.rk4_workspace()

    def norms(Zs):
        c = ol.oracle_constraints(spec, mo.unzip(Zs), O, threads=os.cpu_count())
        return ol.l2_norms(spec, c, bh=BH, radii=RADII)

    hist = [norms(Z)]
    bad = 0
    t0 = time.time()
    for step in range(1, STEPS + 1):
        bad += mo.rk4_step_ws(Z, dt, prm, ws, rhs_fn=ref.lib.ref_bssnRHS_blocks)
        hist.append(norms(Z))
        print(step, hist[-1], f"{time.time() - t0:.0f}s", flush=True)
    idx = sample_nodes(spec.n_nodes)
    np.savez_compressed(
        os.path.join(HERE, "config2_golden.npz"),
        dims=np.array(DIMS), seed=np.array(SEED_MESH), L=np.array(L), origin=np.array(ORIGIN), steps=np.array(STEPS),
        nblocks=np.array(spec.nblocks), zones=np.array(spec.zones()),
        maxabs=np.abs(Z).max(axis=1), sumsq=(Z * Z).sum(axis=1),
        bh=np.array(BH), sample_idx=idx, sample=Z[:, idx], norms=np.array(hist),
        enforce_violations=np.array(bad))


if __name__ == "__main__":
    main()
