"""Regenerates tests/golden/rhs_golden.json from the reference's OWN compiled
CPU arithmetic (oracle/_ref/libbssn_ref.so, built by `make -C oracle` from the
reference sources in place).  Run from the repository root:

    python tests/golden/make_golden.py

Each case is a padded block of Brill-Lindquist data (m = 0.5 punctures at
(+-1, 0, 0)) plus seeded uniform noise, regenerated bit-for-bit from its
parameters by golden_input(); the fixture stores, per variable, the max-norm
and L2 norm of the interior right-hand side and its value at 16 seeded
interior points, all as exact float64 hex strings."""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
import oracle_lib as ol  # noqa: E402

CASES = [
    # side, bflag, h, shift (block pmin + 3h), noise, seed
    (13, 0, 1.0 / 3.0, (0.0, -1.0, -1.0), 1e-8, 1),
    (13, 63, 1.0 / 3.0, (0.5, -1.2, -0.9), 1e-8, 2),
    (13, 1 | 4 | 16, 0.25, (-1.5, -1.5, -1.5), 1e-6, 3),
    (19, 2 | 8 | 32, 0.2, (-1.0, -0.8, -1.1), 1e-8, 4),
    (31, 0, 0.1, (-1.2, -1.4, -1.3), 1e-8, 5),
]


def golden_input(side, h, shift, noise, seed):
    rng = np.random.default_rng(seed)
    n = side ** 3
    pmin = np.array(shift, dtype=np.float64) - 3 * h
    pmax = pmin + (side - 1) * h
    x = pmin[0] + np.arange(side) * h
    y = pmin[1] + np.arange(side) * h
    z = pmin[2] + np.arange(side) * h
    Z, Y, X = np.meshgrid(z, y, x, indexing="ij")
    r1 = np.sqrt((X - 1.0) ** 2 + Y ** 2 + Z ** 2)
    r2 = np.sqrt((X + 1.0) ** 2 + Y ** 2 + Z ** 2)
    with np.errstate(divide="ignore"):
        psi = 1 + 0.5 / (2 * r1) + 0.5 / (2 * r2)
    U = np.zeros((24, n))
    U[0] = np.maximum(1 / psi ** 2, 1e-4).ravel()
    U[1] = np.maximum(1 / psi ** 4, 1e-4).ravel()
    U[12] = U[15] = U[17] = 1.0
    U += noise * rng.uniform(-1, 1, U.shape)
    return U, pmin, pmax


def sample_points(side, seed, k=16):
    rng = np.random.default_rng(1000 + seed)
    pts = []
    for _ in range(k):
        i, j, l = rng.integers(3, side - 3, 3)
        pts.append(int(i + side * (j + side * l)))
    return pts


def interior(R, side):
    return R.reshape(24, side, side, side)[:, 3:-3, 3:-3, 3:-3].reshape(24, -1)


def main():
    ref = ol.reference()
    if ref is None:
        raise SystemExit("oracle/_ref/libbssn_ref.so missing: run `make -C oracle`")
    out = []
    for side, bflag, h, shift, noise, seed in CASES:
        U, pmin, pmax = golden_input(side, h, shift, noise, seed)
        R = ref.bssnrhs(U, 0, pmin, pmax, side, bflag, ol.params())
        Ri = interior(R, side)
        pts = sample_points(side, seed)
        out.append({
            "side": side, "bflag": bflag, "h": h, "shift": list(shift), "noise": noise, "seed": seed,
            "maxnorm": [float(np.abs(Ri[v]).max()).hex() for v in range(24)],
            "l2": [float(np.sqrt((Ri[v] ** 2).sum())).hex() for v in range(24)],
            "points": pts,
            "values": [[float(R[v, p]).hex() for p in pts] for v in range(24)],
        })
    with open(os.path.join(HERE, "rhs_golden.json"), "w") as f:
        json.dump({"source": "reference bssnrhs (BSSN_GR/src/rhs.cpp:80-504 control flow, "
                             "derivs.cpp stencils, bssneqs_eta_const_standard_gauge.cpp) "
                             "compiled with -O2 -ffp-contract=off",
                   "params": "sigma=0.4 lambda={1,1,1,1} lambda_f={1,0} eta=2",
                   "cases": out}, f, indent=1)


if __name__ == "__main__":
    main()
