"""The restatement of G2P on mixed-resolution grids (oracle/msbg_oracle_flip_mr.c)
against the compiled reference, on the CPU.

The fine/coarse distance channel (src/msbg.cpp:1700-1723, 1887-1960,
1994-2029) and its interpolation (SparseGrid::interpolateToFloat<IP_LINEAR>
with OPT_IPBC_NEUMAN, src/sbg.h:3111-3420) come from the reference's own
setRefinementMap and SparseGrid, run through oracle/ref/ref_harness.cpp.  The
velocity blend itself (interpVec3MSBG, src/flip_sim.cpp:1354-1525) is in a
file the reference cannot compile here; on a single-level grid it reduces to
the level-0 restatement, which the last test checks.
"""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from mr_grids import GRIDS, grid_levels, particles_for  # noqa: E402

needs_ref = pytest.mark.skipif(not os.path.exists(oracle.REF_SO),
                               reason="compiled reference not built")

# The reference library is built with FMA contraction (-march=x86-64-v3), the
# restatement without: the interpolated distance (raw units, 1024 per voxel,
# at most 6144) agrees to a few units in the last place.
DIST_INTERP_ATOL = 4e-3


@needs_ref
@pytest.mark.parametrize("name", list(GRIDS))
def test_distance_channel_equals_reference(name):
    res, bsx, nl, lev = grid_levels(name)
    ref = oracle.RefMultires((res,) * 3, bsx, nl, lev)
    try:
        assert ref.dtrans() == 6
        lv_ref, _ = ref.block_info()
        assert (lv_ref == lev).all()
        d_ref, k_ref = ref.dist(nl)
        d, k = oracle.mr_dist([res // bsx] * 3, bsx, lev, nl, ref.dtrans())
        assert (k == k_ref).all()
        assert (d == d_ref).all()
        assert (k == 1).any(), "the grid has fine/coarse transitions"
    finally:
        ref.close()


@needs_ref
@pytest.mark.parametrize("name", list(GRIDS))
def test_distance_interpolation_equals_reference(name):
    res, bsx, nl, lev = grid_levels(name)
    ref = oracle.RefMultires((res,) * 3, bsx, nl, lev)
    try:
        d, k = oracle.mr_dist([res // bsx] * 3, bsx, lev, nl)
        rng = np.random.default_rng(5)
        for lv in range(nl):
            n = res >> lv
            pos = rng.uniform(-1.5, n + 1.5, (40000, 3)).astype(np.float32)
            pos[:2000] = np.round(pos[:2000] * 2) / 2  # on voxel centres and faces
            a = ref.dist_interp(lv, pos)
            b = oracle.mr_dist_interp((res,) * 3, bsx, lev, d, k, lv, pos)
            assert np.abs(a - b).max() <= DIST_INTERP_ATOL, lv
    finally:
        ref.close()


def test_single_level_g2p_equals_level0_restatement():
    res, bsx = 64, 16
    lev = np.zeros((res // bsx) ** 3, np.int32)
    off, n = oracle.mr_layout([res // bsx] * 3, bsx, lev)
    assert n == res ** 3
    rng = np.random.default_rng(3)
    vel = rng.standard_normal(3 * n).astype(np.float32)
    old = rng.standard_normal(3 * n).astype(np.float32)
    p = particles_for(res, 20000, 9)
    d, k = oracle.mr_dist([res // bsx] * 3, bsx, lev, 1)
    assert not d.any() and not k.any()
    a = oracle.mr_g2p((res,) * 3, bsx, lev, p, vel, old, d, k, 0.95)
    b = oracle.flip_g2p(res, bsx, p, vel, old, 0.95)
    assert (a["vel"].view(np.uint32) == b["vel"].view(np.uint32)).all()


def test_layout_offsets():
    res, bsx, nl, lev = grid_levels("z3_b16")
    off, n = oracle.mr_layout([res // bsx] * 3, bsx, lev)
    sizes = (bsx >> lev.astype(np.int64)) ** 3
    assert n == sizes.sum()
    assert (off == np.concatenate([[0], np.cumsum(sizes)[:-1]])).all()


# PressureScene configurations (res, bsx0, nLevels, band): single-level and
# adaptive grids of 8^3, 16^3 and 32^3 blocks
DOWNSAMPLE_CFGS = [(64, 16, 2, 12), (128, 16, 3, 8), (128, 8, 3, 8), (128, 32, 2, 16)]


@needs_ref
@pytest.mark.parametrize("cfg", DOWNSAMPLE_CFGS)
def test_downsample_velocity_equals_reference(cfg):
    """downsampleVelocity restated, bit for bit against the reference on the
    grid its own preparePressureSolveFLIP set up, MG level by MG level."""
    import msbg_gpu
    import ref_pressure as rp

    res, bsx, nl, band = cfg
    R = rp.RefPressure(msbg_gpu.PressureScene(res, bsx, nl, band=band, seed=5))
    try:
        lev0, _ = R.block_levels(0)
        src = np.random.default_rng(1).standard_normal(3 * R.packed_size(0)).astype(np.float32)
        R.set_vec(rp.CH_VEC3_4, src, 0)
        for m in range(1, R.num_levels()):
            lv, _ = R.block_levels(m)
            assert (lv == oracle.mg_levels(lev0, m)).all()
            R.downsample_velocity(m, rp.CH_VEC3_4, rp.CH_VEC3_4)
            ref = R.get_vec(rp.CH_VEC3_4, m)
            flags = R.get(rp.CH_FLAGS, m)
            assert (flags >= 0).all()
            got = oracle.mr_downsample_velocity((res,) * 3, bsx, lev0, m, flags.astype(np.uint16),
                                                src)
            assert (got.view(np.uint32) == ref.view(np.uint32)).all(), m
            src = ref
    finally:
        R.close()
