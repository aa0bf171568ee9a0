"""Regenerates tests/golden/config3_norms.json: the Hamiltonian and momentum
constraint L2 norms (outside r < 0.5 of each puncture) of the batched
workload -- 20,909 blocks of sides 13/19/31/55 drawn with block-count
fractions 0.7/0.2/0.08/0.02 (the seeded split of 10 x 10 x 7 super-cells,
87.0 M zones, spacing 1/30, node (0,0,0) at (-8, -8, -8)), Brill-Lindquist
m1 = m2 = 0.5 at (+-1, 0, 0) plus a seeded 1e-8 perturbation, dt = 0.25 dx,
KO sigma 0.4, eta 2 -- after 0, 2, ..., 10 RK4 steps, evolved on the CPU with
the reference's OWN compiled right-hand side (oracle/_ref, the block loop of
rhs.cpp over bssnrhs) inside the classical RK4 of
BSSN_GR/src/rkBSSN.cpp:764-860 with per-stage constraint enforcement (ghost
fill, zip, stage algebra, enforcement and constraint equations restated in
oracle/bssn_oracle.cpp).  The ghost fill and right-hand side run block by
block (orc_rk4_step_lowmem, bit-identical to the oracle's RK4 step), so the
run needs about 75 GB of host memory instead of 160 GB; 10 steps rather than
the configuration's 100 keep it to about 20 minutes on 16 host cores.  The
mesh comes from the oracle's own generator: the product library is not
loaded.  Run from the repository root:

    python tests/golden/make_config3_golden.py
"""
import json
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import oracle_lib as ol  # noqa: E402

DIMS = (10, 10, 7)
SEED_MESH = 20261203
STEPS = 10
EVERY = 2


def main():
    ref = ol.reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libbssn_ref.so missing: run `make -C oracle REF=...`")
    O = ol.oracle()
    spec = ol.OracleMeshSpec(1, DIMS, seed=SEED_MESH)
    mo = ol.MeshOracle(spec, O)
    prm = ol.params()
    dt = 0.25 * spec.h
    t0 = time.time()
    Z = mo.initial_data(eps=1e-8)
    bufs = [np.empty_like(Z) for _ in range(3)]
    hist = [{"step": 0, "norms": [float(x).hex() for x in ol.constraint_norms_lowmem(spec, Z, O)]}]
    print(0, hist[-1], f"{time.time() - t0:.0f}s", flush=True)
    bad = 0
    for step in range(1, STEPS + 1):
        bad += mo.rk4_step_lowmem(Z, dt, prm, bufs, rhs_fn=ref.lib.ref_bssnRHS_blocks)
        if step % EVERY == 0:
            hist.append({"step": step,
                         "norms": [float(x).hex() for x in ol.constraint_norms_lowmem(spec, Z, O)]})
            print(step, [float.fromhex(x) for x in hist[-1]["norms"]], f"{time.time() - t0:.0f}s",
                  flush=True)
    with open(os.path.join(HERE, "config3_norms.json"), "w") as f:
        json.dump({"workload": "mix20k: 10 x 10 x 7 super-cells, seed 20261203, 20,909 blocks, "
                               "87,036,653 zones, h = 1/30, node (0,0,0) at (-8,-8,-8); "
                               "Brill-Lindquist m=0.5 at (+-1,0,0) + seeded 1e-8 noise; dt = 0.25 dx",
                   "norms": "sqrt(sum c^2 / N) of ham, mom0, mom1, mom2 outside r < 0.5 of each puncture",
                   "nblocks": spec.nblocks, "zones": spec.zones(), "enforce_violations": int(bad),
                   "cpu_seconds": time.time() - t0, "history": hist}, f, indent=1)


if __name__ == "__main__":
    main()
