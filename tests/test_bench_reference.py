"""CPU test of bench.py's reference arm: it times the reference's CPU RK4
step on a mesh from the oracle's own generator and never loads the product
library, and its per-step time is the time it measured."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = """
import runpy, sys
sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'uniform512', '--steps', '2', '--warmup', '0']
runpy.run_path('bench.py', run_name='__main__')
maps = open('/proc/self/maps').read()
print('PRODUCT_LIB_MAPPED', 'libbssn_b200' in maps, 'bssn_b200' in sys.modules)
"""


def test_reference_arm_runs_without_the_product_library():
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.strip().splitlines()
    assert lines[-1] == "PRODUCT_LIB_MAPPED False False", lines[-1]
    out = json.loads(lines[-2])
    assert out["impl"] == "reference"
    assert out["config"]["workload"] == "uniform512" and out["config"]["zones"] == 512 * 343
    assert abs(out["ms_per_step"] - 1e3 * sum(out["step_seconds"]) / 2) < 1e-6
    assert abs(out["value"] - out["config"]["zones"] * 2 / sum(out["step_seconds"])) < 1e-6 * out["value"]
    assert out["cpu_baseline"]["kind"] in ("reference", "port")
    assert out["e2e"]["h2d_bytes_per_step"] == 0


def test_oracle_mesh_generator_matches_the_library():
    """The reference arm's meshes (oracle generator) are the bench's meshes
    (product generator), block for block."""
    sys.path.insert(0, os.path.join(ROOT, "dendro-gr_b200"))
    import numpy as np
    import bssn_b200 as B
    import oracle_lib as ol
    for mode, dims, seed in ((1, (3, 3, 3), 20261203), (0, (8, 8, 8), 0), (1, (2, 1, 3), 7)):
        a = ol.OracleMeshSpec(mode, dims, seed=seed)
        b = B.generate_mesh(mode, dims, seed=seed)
        assert a.G == b.G and a.h == b.h and a.nblocks == b.nblocks
        ba = np.ctypeslib.as_array(a.blocks, shape=(a.nblocks,)).view(np.uint8)
        bb = np.ctypeslib.as_array(b.blocks, shape=(b.nblocks,)).view(np.uint8)
        assert np.array_equal(ba, bb)
