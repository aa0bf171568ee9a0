"""Regenerates tests/golden/constraint_history.json: the Hamiltonian and
momentum constraint L2 norms of the uniform 512-block 13^3 workload
(Brill-Lindquist m=0.5 at (+-1,0,0) on [-8,8]^3 plus seeded 1e-8 noise,
dt = 0.25 dx, KO sigma 0.4, eta 2) every 10 RK4 steps up to 100, evolved
with the reference's OWN compiled right-hand side (oracle/_ref, the block
loop of rhs.cpp over bssnrhs) inside the classical RK4 of
BSSN_GR/src/rkBSSN.cpp:764-860 with per-stage constraint enforcement
(restated in oracle/bssn_oracle.cpp, as are the ghost fill and the
constraint equations).  Run from the repository root:

    python tests/golden/make_constraint_golden.py
"""
import ctypes as C
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "dendro-gr_b200"))
import oracle_lib as ol  # noqa: E402

RK4_C = (1.0 / 6.0, 1.0 / 3.0, 1.0 / 3.0, 1.0 / 6.0)
RK4_U = (0.0, 1.0 / 2.0, 1.0 / 2.0, 1.0)
STEPS, EVERY = 100, 10
RADII = (0.5, 0.5)


def main():
    import bssn_b200 as B  # host-only use: the mesh generator
    ref = ol.reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libbssn_ref.so missing: run `make -C oracle`")
    O = ol.oracle()
    spec = B.generate_mesh(0, (8, 8, 8))
    mo = ol.MeshOracle(spec, O)
    prm = ol.params()
    dt = 0.25 * spec.h
    Z = mo.initial_data()
    O.lib.orc_enforce.restype = C.c_int64

    def rhs(Zs):
        Uz = mo.unzip(Zs)
        R = np.zeros_like(Uz)
        ref.lib.ref_bssnRHS_blocks(ol.rows(R), ol.rows(Uz), spec.blocks, spec.nblocks,
                                   C.byref(prm), 0)
        return mo.zip(R)

    def enforce(Zs):
        return O.lib.orc_enforce(ol.rows(Zs), C.c_int64(spec.n_nodes), C.c_double(1e-4))

    def norms(Zs):
        c = ol.oracle_constraints(spec, mo.unzip(Zs), O)
        return [float(x).hex() for x in ol.l2_norms(spec, c, radii=RADII)]

    hist = [{"step": 0, "norms": norms(Z)}]
    bad = 0
    t0 = time.time()
    for step in range(1, STEPS + 1):
        prev = Z.copy()
        ks = []
        cur = Z
        for s in range(4):
            k = rhs(cur)
            ks.append(k)
            if s < 3:
                im = prev + (RK4_U[s + 1] * dt) * k
                im = np.ascontiguousarray(im)
                bad += enforce(im)
                cur = im
        Z = prev.copy()
        for s in range(4):
            Z += (RK4_C[s] * dt) * ks[s]
        Z = np.ascontiguousarray(Z)
        bad += enforce(Z)
        if step % EVERY == 0:
            hist.append({"step": step, "norms": norms(Z)})
            print(step, [float.fromhex(x) for x in hist[-1]["norms"]], f"{time.time() - t0:.0f}s", flush=True)
    with open(os.path.join(HERE, "constraint_history.json"), "w") as f:
        json.dump({"workload": "uniform 8^3 octree of 13^3 blocks on [-8,8]^3, Brill-Lindquist m=0.5 "
                               "at (+-1,0,0), seeded 1e-8 noise (seed 20261203), dt = 0.25 dx",
                   "norms": "sqrt(sum c^2 / N) of ham, mom0, mom1, mom2 outside r < 0.5 of each puncture",
                   "enforce_violations": int(bad), "history": hist}, f, indent=1)


if __name__ == "__main__":
    main()
