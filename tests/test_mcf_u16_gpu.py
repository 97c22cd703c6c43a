"""Mean-curvature flow on the reference's 16-bit render density.

The reference is built with RenderDensity = uint16_t (RSURF_16_BIT,
src/msbgcell.h:67-68) and its demo smooths that channel
(applyChannelPdeFast<uint16_t>, src/msbg_demo.cpp:716-727, with the [0,1]
clamp): values q stand for q/65535 and are stored back as round(phi*65535)
(src/sbg.h:225-232, 360-368).  The GPU smoother runs on a 16-bit channel
uploaded with msbg_gpu_upload_channel_u16 and is compared with the compiled
reference on the same input, per call: the stencil is FP32 on both sides
with a different operation order, so a voxel may round to the neighbouring
16-bit value; the test bounds that to one quantum in almost every voxel.
"""
import numpy as np
import pytest

import msbg_gpu
import oracle

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_available(), reason="reference not built")]


def density_scene(res, bsx, seed):
    kind, phi = msbg_gpu.sphere_sdf_scene(res, bsx, n_spheres=8, rmin=6, rmax=20, seed=seed)
    dens = np.clip(0.5 - phi / 8.0, 0.0, 1.0)      # density ramp across the surface
    q = np.rint(dens * 65535.0).astype(np.uint16)
    upd = np.nonzero(kind == 1)[0].astype(np.int32)
    return kind, q, upd


@pytest.mark.parametrize("bsx", [8, 16, 32])
def test_u16_mcf_matches_reference_per_call(bsx):
    res = 128
    kind, q, upd = density_scene(res, bsx, seed=31)
    ctx = msbg_gpu.Context(0)
    try:
        ctx.set_topology(res, res, res, bsx)
        ctx.upload_channel_u16(5, 0, kind, q, 0, 65535)
        cur = q.copy()
        for call in range(3):
            ref, _ = oracle.mcf_reference_u16((res,) * 3, bsx, kind, cur, upd, 2, 0.1,
                                              clamp01=True, empty_val=0, full_val=65535)
            ctx.apply_channel_pde_mcf(5, upd, 2, 0.1, clamp01=True)
            got = ctx.download_channel_u16(5, np.empty_like(q))
            d = np.abs(got.astype(np.int64) - ref.astype(np.int64))
            assert d.max() <= 2, (call, int(d.max()))
            assert (d > 0).mean() <= 2e-3, (call, float((d > 0).mean()))
            assert (ref != cur).any()  # the flow moved the surface
            # continue both from the reference's state
            cur = ref
            ctx.upload_channel_u16(5, 0, kind, cur, 0, 65535)
    finally:
        ctx.close()


def test_u16_channel_round_trip_and_type_check():
    res, bsx = 64, 16
    kind, q, upd = density_scene(res, bsx, seed=3)
    ctx = msbg_gpu.Context(0)
    try:
        ctx.set_topology(res, res, res, bsx)
        ctx.upload_channel_u16(1, 0, kind, q, 0, 65535)
        assert (ctx.download_channel_u16(1, np.empty_like(q)) == q).all()
        with pytest.raises(msbg_gpu.MsbgError):  # a 16-bit channel is not an FP32 one
            ctx.download_channel(1, np.empty(q.shape, np.float32))
    finally:
        ctx.close()
