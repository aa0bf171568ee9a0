"""GPU test of the reference-facing C++ drop-in surface
(include/bssn_b200_dendro.hpp) with host arrays: compiled against
libbssn_b200.so and compared with the CPU oracle."""
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as ol

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
LIBDIR = os.path.join(ROOT, "dendro-gr_b200", "lib")


@pytest.fixture(scope="module")
def exe(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("dropin") / "dropin_main")
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "dropin", "dropin_main.cpp"),
                    "-L", LIBDIR, "-lbssn_b200", f"-Wl,-rpath,{LIBDIR}", "-o", out], check=True)
    return out


def test_dropin_bssnrhs_host_arrays(exe, tmp_path):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden as mg
    side, bflag = 19, 42
    U, pmin, pmax = mg.golden_input(side, 0.2, (-1.0, -0.8, -1.1), 1e-8, 77)
    fin, fout = str(tmp_path / "u.bin"), str(tmp_path / "r.bin")
    U.tofile(fin)
    args = [exe, "rhs", str(side), str(bflag)] + [repr(float(x)) for x in pmin] + \
           [repr(float(x)) for x in pmax] + [fin, fout]
    subprocess.run(args, check=True)
    R = np.fromfile(fout).reshape(24, -1)
    ref = ol.oracle().bssnrhs(U, 0, pmin, pmax, side, bflag, ol.params())
    err = ol.rel_err(mg.interior(ref, side), mg.interior(R, side))
    assert err.max() <= 1e-12, err.max()
    # halo of the output untouched (the caller's -7.0 fill)
    cube = R.reshape(24, side, side, side)
    assert (cube[:, :3] == -7.0).all() and (cube[:, :, :, -3:] == -7.0).all()


def test_dropin_stencils_bit_exact(exe, tmp_path):
    side = 13
    rng = np.random.default_rng(4)
    u = 1.0 + 1e-8 * rng.standard_normal(side ** 3)
    fin, fout = str(tmp_path / "u.bin"), str(tmp_path / "d.bin")
    u.tofile(fin)
    O = ol.oracle()
    for kind in range(9):
        for bflag in (0, 63, 5):
            subprocess.run([exe, "deriv", str(kind), str(side), str(bflag), "0.3", fin, fout], check=True)
            got = np.fromfile(fout)
            ref = O.stencil(kind, u, 0.3, (side, side, side), bflag)
            assert np.array_equal(got.view(np.uint64), ref.view(np.uint64)), (kind, bflag)


def test_dropin_reference_signatures(exe, tmp_path):
    """The reference's own argument lists (rhs.h:28-36 with t and
    uZipConstVars, bssn_constraints.h:15 per node): bssnrhs and the
    block-list bssnRHS over a stand-in ot::Block agree bit for bit, match the
    oracle at 1e-12, and per-node enforcement matches the oracle's."""
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests", "golden"))
    import make_golden as mg
    side, bflag = 13, 21
    U, _, _ = mg.golden_input(side, 0.25, (-1.0, -0.8, -1.1), 1e-8, 91)
    fin, frhs, fenf = (str(tmp_path / f) for f in ("u.bin", "r.bin", "e.bin"))
    U.tofile(fin)
    subprocess.run([exe, "refsig", str(side), str(bflag), fin, frhs, fenf], check=True)
    raw = np.fromfile(frhs)
    R, pmin, pmax = raw[:-6].reshape(24, -1), raw[-6:-3], raw[-3:]
    ref = ol.oracle().bssnrhs(U, 0, pmin, pmax, side, bflag, ol.params())
    err = ol.rel_err(mg.interior(ref, side), mg.interior(R, side))
    assert err.max() <= 1e-12, err.max()
    E = np.fromfile(fenf).reshape(24, -1)
    want = U.copy()
    assert ol.oracle().enforce(want, 1e-4) == 0
    assert ol.rel_err(want, E).max() <= 1e-14
