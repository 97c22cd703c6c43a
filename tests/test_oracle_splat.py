"""The CPU restatement of the particle splatting, pinned to the reference.

The fixtures under tests/golden/splat_*.npz come from the reference's own
demo, msbg_test_sparse (src/msbg_demo.cpp), run through
oracle/ref/splat_harness.cpp (tests/golden/make_splat_golden.py): its
particles, its value blocks, the quantised squared distances after its splat
loop and the render density after its finalisation.  The restatement
(oracle/msbg_oracle_splat.c) must reproduce every value exactly.
"""
import math
import os

import numpy as np
import pytest

import oracle

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["splat_demo_b8", "splat_demo_b16", "splat_demo_b32"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


@pytest.mark.parametrize("name", CASES)
def test_oracle_reproduces_reference_demo(name):
    g = load(name)
    res3, bsx = tuple(int(v) for v in g["res"]), int(g["bsx"])
    act = oracle.splat_mark(res3, bsx, g["pos"])
    assert np.array_equal(np.nonzero(act)[0], g["blocks"])
    raw = oracle.splat(res3, bsx, act, g["pos"], finalize=False)
    assert np.array_equal(raw, g["raw"])
    fin = oracle.splat(res3, bsx, act, g["pos"], finalize=True)
    assert np.array_equal(fin, g["final"])
    # the fixture is not trivial: most particles splat, values span the range
    assert (g["raw"] < 65535).sum() > 1000 and g["final"].max() > 60000


def test_domain_test_matches_reference():
    g = load("splat_domain")
    res3 = tuple(int(v) for v in g["res"])
    lo, hi = oracle.splat_domain(res3)
    p = g["pts"]
    with np.errstate(invalid="ignore"):
        keep = np.isfinite(p).all(1) & ~((p < lo) | (p > hi)).any(1)
    assert np.array_equal(keep.astype(np.int32), g["keep"])
    # the probes straddle the bounds: both outcomes occur on every axis
    assert 0 < g["keep"].sum() < len(g["keep"])


def literal_splat(res3, bsx, kind, pos, r_particle, nb_dist):
    """The demo's splat loop (src/msbg_demo.cpp:553-636) written out in
    Python floats for a handful of particles: double-precision distances,
    so only the goto/continue structure is compared, on voxels far from
    rounding ties."""
    nbx, nby = res3[0] // bsx, res3[1] // bsx
    slot = np.cumsum(kind == 1) - 1
    out = np.full(int((kind == 1).sum()) * bsx ** 3, 65535, np.int64)
    r_scan = r_particle + nb_dist
    dmax = r_scan * r_scan
    for p in pos:
        c = [int(v) for v in p]
        b = c[0] // bsx + nbx * (c[1] // bsx + nby * (c[2] // bsx))
        if kind[b] != 1:
            continue
        lo = [max(math.ceil(v - r_scan - 0.5), 0) for v in p]
        hi = [min(math.floor(v + r_scan - 0.5), s - 1) for v, s in zip(p, res3)]
        done = False
        for iz in range(lo[2], hi[2] + 1):
            for iy in range(lo[1], hi[1] + 1):
                for ix in range(lo[0], hi[0] + 1):
                    d = (ix - p[0] + 0.5) ** 2 + (iy - p[1] + 0.5) ** 2 + (iz - p[2] + 0.5) ** 2
                    if d > dmax:
                        continue
                    vb = ix // bsx + nbx * (iy // bsx + nby * (iz // bsx))
                    if kind[vb] != 1:
                        done = True
                        break
                    i = slot[vb] * bsx ** 3 + ix % bsx + bsx * (iy % bsx + bsx * (iz % bsx))
                    out[i] = min(out[i], int(math.floor(d / dmax * 65535 + 0.5)))
                if done:
                    break
            if done:
                break
    return out


def test_scan_stops_at_the_first_block_without_values():
    """Particles next to blocks without values: the scan ends at the first
    voxel in such a block (the demo's goto loop_exit)."""
    res3, bsx = (32, 32, 32), 8
    nb = (res3[0] // bsx) ** 3
    kind = np.ones(nb, np.int8)
    kind[[1, 5, 21, 22, 42]] = 2  # const empty blocks among the value blocks
    pos = np.array([[7.25, 2.5, 3.75], [9.125, 9.5, 10.5], [20.375, 22.25, 12.5],
                    [15.5, 15.5, 15.5], [4.0625, 17.75, 30.5]], np.float32)
    got = oracle.splat(res3, bsx, kind, pos, finalize=False).astype(np.int64)
    want = literal_splat(res3, bsx, kind, pos.astype(np.float64), 2.0, 2.0)
    assert np.abs(got - want).max() <= 1
    # the stop matters here: a scan without it writes more voxels
    full = literal_splat(res3, bsx, np.ones(nb, np.int8), pos.astype(np.float64), 2.0, 2.0)
    keep = np.repeat(kind == 1, bsx ** 3)
    assert (full[keep] < 65535).sum() > (got < 65535).sum()


def test_finalisation_table():
    t = oracle.splat_finalize_table(2.0, 2.0).astype(np.int64)
    assert t[0] == 65535                      # at the particle centre
    assert (np.diff(t) <= 0).all()            # farther is lower
    assert (t[int(0.999 * 65535) + 1:] == 0).all()
    # the ramp runs from d - rParticle = -rParticle (1) to rParticle + nbDist
    # (0): d = 3 lies half way
    q = int(round((3.0 / 4.0) ** 2 * 65535))
    assert abs(t[q] - 65535 * 0.5) <= 2


@pytest.mark.skipif(not oracle.splat_reference_available(), reason="reference not built")
def test_oracle_matches_live_reference(tmp_path):
    """A fresh seeded base cloud run through the reference demo here."""
    rng = np.random.default_rng(77)
    v = rng.normal(size=(36, 3))
    ply = str(tmp_path / "base.ply")
    oracle.write_ply(ply, v)
    r = oracle.splat_reference_demo(ply, 1, 16, (96, 96, 96))
    act = oracle.splat_mark((96,) * 3, 16, r["pos"])
    assert np.array_equal(np.nonzero(act)[0], r["blocks"])
    assert np.array_equal(oracle.splat((96,) * 3, 16, act, r["pos"]), r["final"])
