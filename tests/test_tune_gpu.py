"""GPU tests of the autotuner and its cache: the FP64 cube operator's stage
tile widths are timed once and stored under a key of the device, the points
per axis and the quadrature count; a cache file is appended to, read back by
a new process, and an entry in it decides the tiles without timing."""
import os
import subprocess
import sys

import numpy as np
import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CHILD = r"""
import sys
sys.path.insert(0, {root!r})
import dage_b200 as dage
dage.set_tune_cache({path!r})
g = dage.Grid3D.cube(-3.0, 5, 0.2)
op = dage.Coulomb3D(g, quad=dage.GaussQuad(6, 6))
print("TILES", *op.tiles)
"""


def _child(path):
    out = subprocess.run([sys.executable, "-c", CHILD.format(root=ROOT, path=path)],
                         capture_output=True, text=True, timeout=300)
    assert out.returncode == 0, out.stderr
    line = [l for l in out.stdout.splitlines() if l.startswith("TILES")][0]
    return tuple(int(x) for x in line.split()[1:])


def test_tune_cache_file_round_trip(tmp_path):
    path = str(tmp_path / "tune.txt")
    tiles = _child(path)  # tunes and appends
    assert all(t in (32, 64, 128) for t in tiles)
    lines = open(path).read().splitlines()
    key = [l for l in lines if "/op3d_fp64/31x31,31x31,31x31,P12" in l]
    assert key, lines
    # an edited entry decides the tiles of a new process (no timing)
    forced = (32, 128, 64)
    with open(path, "a") as f:
        f.write(key[-1].split()[0] + " %d %d %d\n" % forced)
    assert _child(path) == forced


def test_tuned_tiles_give_the_same_potential(dage, oracle):
    g = dage.Grid3D.cube(-12.0, 20, 0.2)
    go = oracle.Grid3D.cube(-12.0, 20, 0.2)
    rng = np.random.default_rng(4)
    rho = oracle.gauss_cube(go, rng.uniform(0.5, 2, 2), rng.uniform(0.5, 4, 2),
                            rng.uniform(-3, 3, (2, 3)))
    op = dage.Coulomb3D(g, quad=dage.GaussQuad(20, 20))
    print("121^3 tiles", op.tiles)
    V, E = op.apply(rho, energy=True)
    Vo = oracle.coulomb_apply(go, rho, quad=(20, 20, 0.0, 2.0, 1e3))
    assert np.abs(V - Vo).max() <= 1e-10 * np.abs(Vo).max()
