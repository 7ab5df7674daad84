"""GPU tests of the autotuner and its cache: the FP64 cube operator's stage
tile widths and the split-precision operator's tensor-core schedule are
timed once and stored under a key of the device, the points per axis and the
quadrature count; a cache file is appended to, read back by a new process,
and an entry in it decides the choice without timing."""
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


def test_operator_cache_on_disk(dage, oracle, tmp_path):
    """dage_op3d_create_cached writes the matrices on the first create and
    reads them on the next (same grids and quadrature: identical potential,
    bit for bit); another quadrature is another key."""
    g = dage.Grid3D.cube(-3.0, 5, 0.2)
    go = oracle.Grid3D.cube(-3.0, 5, 0.2)
    rho = oracle.gauss_cube(go, [1.0, -0.5], [1.2, 2.5], [[0.1, 0.2, -0.3], [-0.4, 0.0, 0.5]])
    q = dage.GaussQuad(8, 8)
    d = str(tmp_path)
    a = dage.Coulomb3D(g, quad=q, cache_dir=d)
    assert not a.from_cache
    files = os.listdir(d)
    assert len(files) == 1 and files[0].startswith("op3d_") and files[0].endswith(".bin")
    b = dage.Coulomb3D(g, quad=q, cache_dir=d)
    assert b.from_cache
    Va, Ea = a.apply(rho, energy=True)
    Vb, Eb = b.apply(rho, energy=True)
    assert np.array_equal(Va, Vb) and Ea == Eb
    for k in range(3):  # the stored matrices are the built ones
        assert np.array_equal(a.matrix(k), b.matrix(k))
    c = dage.Coulomb3D(g, quad=dage.GaussQuad(6, 6), cache_dir=d)
    assert not c.from_cache and len(os.listdir(d)) == 2
    m = dage.Coulomb3D(g, quad=q, cache_dir=d, precision="fp16x3")  # mixed ops read it too
    assert m.from_cache


MIXED_CHILD = r"""
import sys
import numpy as np
sys.path.insert(0, {root!r})
import dage_b200 as dage
from oracle import oracle as O
dage.set_tune_cache({path!r})
g = dage.Grid3D.cube(-6.0, 10, 0.2)
go = O.Grid3D.cube(-6.0, 10, 0.2)
rho = O.gauss_cube(go, [1.0, 0.6], [1.5, 3.0], [[0.3, -0.2, 0.1], [-0.9, 0.8, 0.4]])
op = dage.Coulomb3D(g, quad=dage.GaussQuad(10, 10), precision="fp16x3")
V, E = op.apply(rho, energy=True)
np.save({out!r}, np.concatenate([V.reshape(-1, order="F"), [E]]))
print("SCHEDULE", *op.schedule)
"""


def _mixed_child(path, out):
    r = subprocess.run([sys.executable, "-c", MIXED_CHILD.format(root=ROOT, path=path, out=out)],
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    line = [l for l in r.stdout.splitlines() if l.startswith("SCHEDULE")][0]
    return tuple(int(x) for x in line.split()[1:]), np.load(out)


def test_mixed_schedule_tuned_and_forced(dage, oracle, tmp_path):
    """The tensor-core schedule (ring stages, t-points per last-stage pass)
    is timed once and cached (the ring depth; the group stays at min(P, 8)
    so that results do not depend on a timing); an edited entry forces
    another schedule in a new process, and every schedule gives the same
    potential to the split-precision bars (the ring depth changes no
    arithmetic, the group only the order of the last stage's FP32 sums)."""
    path = str(tmp_path / "tune.txt")
    sched, ref = _mixed_child(path, str(tmp_path / "a.npy"))
    assert sched[0] in (4, 6) and sched[1] == 8
    key = [l for l in open(path).read().splitlines() if "/op3d_mixed3/61x61,61x61,61x61,P20" in l]
    assert key
    for forced in ((4, 4), (6, 8), (4, 8)):
        with open(path, "a") as f:
            f.write(key[-1].split()[0] + " %d %d\n" % forced)
        got, res = _mixed_child(path, str(tmp_path / "b.npy"))
        assert got == forced
        V, Vr = res[:-1], ref[:-1]
        assert np.abs(V - Vr).max() <= 2e-7 * np.abs(Vr).max()
        assert abs(res[-1] - ref[-1]) <= 5e-8 * abs(ref[-1])
        if forced[1] == sched[1]:
            assert np.array_equal(res, ref)  # same group: identical sums
