"""G2P on mixed-resolution grids on the GPU (msbg_gpu_flip_mr_dist,
msbg_gpu_flip_mr_channel, msbg_gpu_flip_g2p_mr[_device]) against the CPU
restatement, which tests/test_oracle_flip_mr.py pins to the compiled
reference where the reference compiles: the distance channel bit for bit,
the particle velocities bit for bit (both evaluate the reference's
expressions in its order without contraction)."""
import os
import sys

import numpy as np
import pytest

import msbg_gpu
import oracle

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
from mr_grids import GRIDS, grid_levels, particles_for  # noqa: E402

pytestmark = pytest.mark.gpu

ALPHA = 0.95


def _ctx(name):
    res, bsx, nl, lev = grid_levels(name)
    ctx = msbg_gpu.Context(0)
    ctx.set_topology(res, res, res, bsx, nl, lev)
    return ctx, res, bsx, nl, lev


def _channels(n, seed):
    rng = np.random.default_rng(seed)
    return (rng.standard_normal(3 * n).astype(np.float32),
            rng.standard_normal(3 * n).astype(np.float32))


@pytest.mark.parametrize("name", list(GRIDS))
def test_distance_channel_bit_identical(name):
    ctx, res, bsx, nl, lev = _ctx(name)
    try:
        d, k = ctx.flip_mr_dist(nl)
        d_o, k_o = oracle.mr_dist([res // bsx] * 3, bsx, lev, nl)
        assert (k == k_o).all()
        assert (d == d_o).all()
        if os.path.exists(oracle.REF_SO):  # the compiled reference, where it was built
            ref = oracle.RefMultires((res,) * 3, bsx, nl, lev)
            d_r, k_r = ref.dist(nl)
            ref.close()
            assert (k == k_r).all() and (d == d_r).all()
    finally:
        ctx.close()


@pytest.mark.parametrize("name", list(GRIDS))
def test_g2p_bit_identical_to_restatement(name):
    ctx, res, bsx, nl, lev = _ctx(name)
    try:
        n = msbg_gpu.packed_voxels(bsx, lev)
        vel, old = _channels(n, 1)
        ctx.flip_mr_channel(msbg_gpu.FLIP_VEL, vel)
        ctx.flip_mr_channel(msbg_gpu.FLIP_VEL_OLD, old)
        assert (ctx.flip_mr_channel(msbg_gpu.FLIP_VEL) == vel).all()
        p = particles_for(res, 200_000, 2)
        q = p.copy()
        ctx.flip_g2p_mr(q, ALPHA)
        d, k = oracle.mr_dist([res // bsx] * 3, bsx, lev, nl)
        e = oracle.mr_g2p((res,) * 3, bsx, lev, p, vel, old, d, k, ALPHA)
        assert (q["pos"].view(np.uint32) == p["pos"].view(np.uint32)).all()
        assert (q["vel"].view(np.uint32) == e["vel"].view(np.uint32)).all()
        # coarse blocks were reached and blended
        assert (lev > 0).any()
    finally:
        ctx.close()


def test_g2p_device_particles_equal_host_particles():
    import torch

    ctx, res, bsx, nl, lev = _ctx("z3_b16")
    try:
        n = msbg_gpu.packed_voxels(bsx, lev)
        vel, old = _channels(n, 4)
        ctx.flip_mr_channel(msbg_gpu.FLIP_VEL, vel)
        ctx.flip_mr_channel(msbg_gpu.FLIP_VEL_OLD, old)
        p = particles_for(res, 50_000, 6)
        q = p.copy()
        ctx.flip_g2p_mr(q, ALPHA)
        dev = torch.from_numpy(p.view(np.uint8).copy()).to("cuda:0")
        ctx.flip_g2p_mr_device(dev.data_ptr(), len(p), ALPHA)
        got = dev.cpu().numpy().view(msbg_gpu.FLIP_PARTICLE)
        assert (got["vel"].view(np.uint32) == q["vel"].view(np.uint32)).all()
    finally:
        ctx.close()


def test_single_level_g2p_equals_level0_entry_point():
    res, bsx = 64, 16
    ctx = msbg_gpu.Context(0)
    try:
        ctx.set_topology(res, res, res, bsx)
        n = res ** 3
        vel, old = _channels(n, 8)
        ctx.flip_channel(msbg_gpu.FLIP_VEL, n, vel)
        ctx.flip_channel(msbg_gpu.FLIP_VEL_OLD, n, old)
        ctx.flip_mr_channel(msbg_gpu.FLIP_VEL, vel)
        ctx.flip_mr_channel(msbg_gpu.FLIP_VEL_OLD, old)
        p = particles_for(res, 50_000, 10)
        a, b = p.copy(), p.copy()
        ctx.flip_g2p(a, ALPHA)
        ctx.flip_g2p_mr(b, ALPHA)
        assert (a["vel"].view(np.uint32) == b["vel"].view(np.uint32)).all()
    finally:
        ctx.close()


def test_topology_change_rebuilds_and_bad_inputs_are_rejected():
    ctx, res, bsx, nl, lev = _ctx("sphere2_b8")
    try:
        d0, _ = ctx.flip_mr_dist(nl)
        # a different level map on the same grid gives its own channel
        lev2 = np.zeros_like(lev)
        lev2[: len(lev) // 2] = 1
        ctx.set_topology(res, res, res, bsx, nl, lev2)
        d1, k1 = ctx.flip_mr_dist(nl)
        d_o, k_o = oracle.mr_dist([res // bsx] * 3, bsx, lev2, nl)
        assert (d1 == d_o).all() and (k1 == k_o).all()
        # neighbours two levels apart: rejected as the reference's assertion does
        bad = np.zeros_like(lev)
        bad[0] = 2
        ctx.set_topology(res, res, res, bsx, 3, bad)
        with pytest.raises(msbg_gpu.MsbgError):
            ctx.flip_mr_dist(3)
        ctx.set_topology(res, res, res, bsx, nl, lev)
        with pytest.raises(msbg_gpu.MsbgError):  # wrong channel size
            ctx.flip_mr_channel(msbg_gpu.FLIP_VEL, np.zeros(5, np.float32))
        with pytest.raises(msbg_gpu.MsbgError):  # no such channel
            ctx.flip_mr_channel(msbg_gpu.FLIP_MASS, np.zeros(3 * msbg_gpu.packed_voxels(bsx, lev),
                                                            np.float32))
        ctx.flip_g2p_mr(np.zeros(0, msbg_gpu.FLIP_PARTICLE))  # no particles: nothing to do
    finally:
        ctx.close()


def test_large_grid_sampled_against_restatement():
    """512^3, 16^3 blocks, 3 levels around a seeded sphere; 8 M particles on
    the GPU, a seeded sample of 400 k checked bit for bit."""
    res, bsx, nl = 512, 16, 3
    nb = res // bsx
    b = np.arange(nb ** 3)
    bx, by, bz = b % nb, (b // nb) % nb, b // (nb * nb)
    r = np.sqrt((bx - 12.5) ** 2 + (by - 15.5) ** 2 + (bz - 17.5) ** 2)
    lev = np.where(r < 7, 0, np.where(r < 12, 1, 2)).astype(np.int32)
    ctx = msbg_gpu.Context(0)
    try:
        ctx.set_topology(res, res, res, bsx, nl, lev)
        n = msbg_gpu.packed_voxels(bsx, lev)
        vel, old = _channels(n, 12)
        ctx.flip_mr_channel(msbg_gpu.FLIP_VEL, vel)
        ctx.flip_mr_channel(msbg_gpu.FLIP_VEL_OLD, old)
        p = particles_for(res, 8_000_000, 13, margin=0.5)
        q = p.copy()
        ctx.flip_g2p_mr(q, ALPHA)
        idx = np.random.default_rng(14).choice(len(p), 400_000, replace=False)
        d, k = oracle.mr_dist([nb] * 3, bsx, lev, nl)
        e = oracle.mr_g2p((res,) * 3, bsx, lev, p[idx], vel, old, d, k, ALPHA)
        assert (q["vel"][idx].view(np.uint32) == e["vel"].view(np.uint32)).all()
    finally:
        ctx.close()


@pytest.mark.parametrize("cfg", [(64, 16, 2, 12), (128, 16, 3, 8), (128, 8, 3, 8),
                                 (128, 32, 2, 16)])
def test_downsample_velocity_bit_identical(cfg):
    """msbg_gpu_flip_downsample_velocity against the restatement (pinned bit
    for bit to the reference's downsampleVelocity on the CPU), MG level by MG
    level, with the cell flags of the reference's own prepare where the
    compiled reference is present, else SOLID/VOID flags of a seeded mix."""
    res, bsx, nl, band = cfg
    scene = msbg_gpu.PressureScene(res, bsx, nl, band=band, seed=5)
    lev0 = np.ascontiguousarray(scene.block_levels, np.int32)
    ref = None
    if os.path.exists(oracle.REF_SO):
        import ref_pressure as rp
        ref = rp.RefPressure(scene)
    ctx = msbg_gpu.Context(0)
    try:
        ctx.set_topology(res, res, res, bsx, nl, lev0)
        rng = np.random.default_rng(2)
        _, n0 = oracle.mr_layout([res // bsx] * 3, bsx, lev0)
        src = rng.standard_normal(3 * n0).astype(np.float32)
        if ref is not None:
            ref.set_vec(rp.CH_VEC3_4, src, 0)
        for m in range(1, nl):
            _, nm = oracle.mr_layout([res // bsx] * 3, bsx, oracle.mg_levels(lev0, m))
            if ref is not None:
                flags = ref.get(rp.CH_FLAGS, m).astype(np.uint16)
            else:
                flags = rng.choice(np.array([0, 0, 0, 1, 0x1000], np.uint16), nm)
            got = ctx.flip_downsample_velocity(m, flags, src)
            exp = oracle.mr_downsample_velocity((res,) * 3, bsx, lev0, m, flags, src)
            assert (got.view(np.uint32) == exp.view(np.uint32)).all(), m
            if ref is not None:
                ref.downsample_velocity(m, rp.CH_VEC3_4, rp.CH_VEC3_4)
                assert (got.view(np.uint32) == ref.get_vec(rp.CH_VEC3_4, m).view(np.uint32)).all()
            src = got
        with pytest.raises(msbg_gpu.MsbgError):  # MG level 0 has no finer source
            ctx.flip_downsample_velocity(0, np.zeros(n0, np.uint16), src)
    finally:
        ctx.close()
        if ref is not None:
            ref.close()
