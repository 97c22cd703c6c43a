"""CPU tests of the smoother oracle: pinned to the compiled reference."""
import glob
import os

import numpy as np
import pytest

import oracle
from conftest import GOLDEN

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "mcf_*.npz")))


def tol_ok(a, b, rel=1e-5):
    """FP32 parity bar of the smoother: |a-b| <= rel * max(1, |b|) everywhere."""
    return np.all(np.abs(a - b) <= rel * np.maximum(1.0, np.abs(b)))


def load(f):
    z = np.load(f)
    res3 = tuple(int(v) for v in z["res3"])
    bsx = int(z["bsx"])
    nb3 = tuple(r // bsx for r in res3)
    return z, res3, bsx, nb3


@pytest.mark.parametrize("f", FIXTURES, ids=[os.path.basename(f) for f in FIXTURES])
@pytest.mark.parametrize("iters", [2, 20])
def test_oracle_matches_golden(f, iters):
    z, res3, bsx, nb3 = load(f)
    out = oracle.mcf_oracle(nb3, bsx, z["kind"], z["values"], z["update"], iters, float(z["dt"]),
                            bool(z["clamp01"]), float(z["empty_val"]), float(z["full_val"]))
    assert tol_ok(out, z[f"out{iters}"])


def test_fixtures_exist():
    assert len(FIXTURES) >= 3


def test_odd_iteration_count_rounds_up_to_even():
    z, res3, bsx, nb3 = load(FIXTURES[0])
    a = oracle.mcf_oracle(nb3, bsx, z["kind"], z["values"], z["update"], 1, 0.1)
    b = oracle.mcf_oracle(nb3, bsx, z["kind"], z["values"], z["update"], 2, 0.1)
    np.testing.assert_array_equal(a, b)


def test_constant_and_linear_fields_are_fixed_points():
    nb3, bsx = (2, 2, 2), 8
    kind = np.ones(8, np.int8)
    upd = np.arange(8, dtype=np.int32)
    const = np.full((8, bsx, bsx, bsx), 2.5, np.float32)
    out = oracle.mcf_oracle(nb3, bsx, kind, const, upd, 4, 0.1, empty_val=2.5, full_val=2.5)
    np.testing.assert_array_equal(out, const)
    # linear field in z: Neumann clamps at the domain boundary are the only curvature
    lin = np.empty_like(const)
    for b in range(8):
        bz = b // 4
        lin[b] = (bz * bsx + np.arange(bsx, dtype=np.float32))[:, None, None]
    out = oracle.mcf_oracle(nb3, bsx, kind, lin, upd, 2, 0.1)
    np.testing.assert_array_equal(out, lin)


def test_same_colour_blocks_never_touch():
    nbx = nby = nbz = 6
    col = {}
    for bz in range(nbz):
        for by in range(nby):
            for bx in range(nbx):
                col[(bx, by, bz)] = (bx & 1) + 2 * (by & 1) + 4 * (bz & 1)
    for (bx, by, bz), c in col.items():
        for dz in (-1, 0, 1):
            for dy in (-1, 0, 1):
                for dx in (-1, 0, 1):
                    if dx == dy == dz == 0:
                        continue
                    n = (bx + dx, by + dy, bz + dz)
                    if n in col:
                        assert col[n] != c


@pytest.mark.skipif(not oracle.ref_available(), reason="compiled reference not built")
def test_oracle_matches_compiled_reference_on_sphere_scene():
    import msbg_gpu
    res, bsx = 96, 16
    kind, vals = msbg_gpu.sphere_sdf_scene(res, bsx, n_spheres=6, rmin=8, rmax=20, band=4, seed=3)
    upd = np.nonzero(kind == 1)[0].astype(np.int32)
    o = oracle.mcf_oracle((res // bsx,) * 3, bsx, kind, vals, upd, 6, 0.1)
    r, _ = oracle.mcf_reference((res,) * 3, bsx, kind, vals, upd, 6, 0.1)
    assert tol_ok(o, r)
    assert np.abs(r - vals).max() > 0.05  # the smoother did change the field
