"""GPU parity of the 8-colour mean-curvature-flow smoother (through the C ABI)."""
import glob
import os

import numpy as np
import pytest

import msbg_gpu
import oracle
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

FIXTURES = sorted(glob.glob(os.path.join(GOLDEN, "mcf_*.npz")))
CH = 7  # any channel id


def tol_ok(a, b, rel=1e-5):
    """FP32 parity bar: |gpu - ref| <= 1e-5 * max(1, |ref|) at every voxel."""
    err = np.abs(a - b) / np.maximum(1.0, np.abs(b))
    return err.max() <= rel, float(err.max())


def run_gpu(ctx, res3, bsx, kind, vals, upd, iters, dt=0.1, clamp01=False, ev=4.0, fv=-4.0,
            calls=1):
    ctx.set_topology(*res3, bsx)
    ctx.upload_channel(CH, 0, kind, vals, ev, fv)
    outs = []
    for _ in range(calls):
        ctx.apply_channel_pde_mcf(CH, upd, iters, dt, clamp01)
        outs.append(ctx.download_channel(CH, np.empty_like(vals)))
    return outs


@pytest.mark.parametrize("f", FIXTURES, ids=[os.path.basename(f) for f in FIXTURES])
def test_gpu_matches_reference_golden(gpu_ctx, f):
    z = np.load(f)
    res3 = tuple(int(v) for v in z["res3"])
    bsx = int(z["bsx"])
    o2, o20 = None, None
    outs = run_gpu(gpu_ctx, res3, bsx, z["kind"], z["values"], z["update"], 2, float(z["dt"]),
                   bool(z["clamp01"]), float(z["empty_val"]), float(z["full_val"]), calls=10)
    ok2, e2 = tol_ok(outs[0], z["out2"])
    ok20, e20 = tol_ok(outs[-1], z["out20"])
    assert ok2, e2
    assert ok20, e20
    # blocks not in the update list are read but never written
    kind = z["kind"]
    vid = np.nonzero(kind == 1)[0]
    frozen = ~np.isin(vid, z["update"])
    np.testing.assert_array_equal(outs[-1][frozen], z["values"][frozen])


@pytest.mark.parametrize("bsx", [8, 16, 32])
def test_gpu_per_call_parity_with_oracle(gpu_ctx, bsx):
    res = 128
    kind, vals = msbg_gpu.sphere_sdf_scene(res, bsx, n_spheres=10, rmin=10, rmax=30, seed=21 + bsx)
    upd = np.nonzero(kind == 1)[0].astype(np.int32)
    outs = run_gpu(gpu_ctx, (res,) * 3, bsx, kind, vals, upd, 2, calls=10)
    ref = vals
    for k, out in enumerate(outs):
        ref = oracle.mcf_oracle((res // bsx,) * 3, bsx, kind, ref, upd, 2, 0.1)
        ok, e = tol_ok(out, ref)
        assert ok, (k, e)
        ref = out  # compare each call from the same starting state


def test_gpu_block_pointer_upload_equals_packed(gpu_ctx):
    res, bsx = 64, 16
    kind, vals = msbg_gpu.sphere_sdf_scene(res, bsx, n_spheres=3, rmin=8, rmax=16, seed=2)
    kind = kind.copy()
    kind[kind == 2] = 0  # NULL blocks -> Neumann halo
    upd = np.nonzero(kind == 1)[0].astype(np.int32)
    gpu_ctx.set_topology(res, res, res, bsx)
    blocks = [None] * len(kind)
    it = iter(vals)
    for b in range(len(kind)):
        if kind[b] == 1:
            blocks[b] = next(it)
    gpu_ctx.upload_channel_blocks(CH, 0, kind, blocks, 4.0, -4.0)
    gpu_ctx.apply_channel_pde_mcf(CH, upd, 4, 0.1)
    a = gpu_ctx.download_channel(CH, np.empty_like(vals))
    (b,) = run_gpu(gpu_ctx, (res,) * 3, bsx, kind, vals, upd, 4)
    np.testing.assert_array_equal(a, b)
    ref = oracle.mcf_oracle((res // bsx,) * 3, bsx, kind, vals, upd, 4, 0.1)
    assert tol_ok(a, ref)[0]


def test_gpu_full_size_sphere_band_512(gpu_ctx):
    """512^3, 16^3 blocks, 64 spheres, band 4, 20 iterations, dt 0.1."""
    res, bsx = 512, 16
    kind, vals = msbg_gpu.sphere_sdf_scene(res, bsx, n_spheres=64, rmin=20, rmax=60, band=4,
                                           seed=1234)
    upd = np.nonzero(kind == 1)[0].astype(np.int32)
    (out,) = run_gpu(gpu_ctx, (res,) * 3, bsx, kind, vals, upd, 20)
    # size-independent properties: each iteration moves a voxel by at most 0.1
    assert np.abs(out - vals).max() <= 20 * 0.1 + 1e-4
    assert np.isfinite(out).all()
    ref = oracle.mcf_oracle((res // bsx,) * 3, bsx, kind, vals, upd, 20, 0.1)
    ok, e = tol_ok(out, ref)
    assert ok, e


def test_gpu_rejects_non_value_block_in_list(gpu_ctx):
    res, bsx = 64, 16
    kind, vals = msbg_gpu.sphere_sdf_scene(res, bsx, n_spheres=3, rmin=8, rmax=16, seed=2)
    kind = kind.copy()
    kind[5] = 2  # make block 5 a const block
    vals = vals[:int((kind == 1).sum())]
    gpu_ctx.set_topology(res, res, res, bsx)
    gpu_ctx.upload_channel(CH, 0, kind, vals, 4.0, -4.0)
    bad = np.array([5], np.int32)
    with pytest.raises(msbg_gpu.MsbgError) as ei:
        gpu_ctx.apply_channel_pde_mcf(CH, bad, 2, 0.1)
    assert ei.value.code == 5
    with pytest.raises(msbg_gpu.MsbgError):
        gpu_ctx.apply_channel_pde_mcf(CH, np.array([len(kind)], np.int32), 2, 0.1)


def test_gpu_constant_field_is_fixed_point(gpu_ctx):
    res, bsx = 32, 16
    kind = np.ones(8, np.int8)
    vals = np.full((8, bsx, bsx, bsx), 1.25, np.float32)
    (out,) = run_gpu(gpu_ctx, (res,) * 3, bsx, kind, vals, np.arange(8, dtype=np.int32), 6,
                     ev=1.25, fv=1.25)
    np.testing.assert_array_equal(out, vals)


def test_reupload_reuses_and_resizes_the_channel(gpu_ctx):
    """A channel uploaded again under the same id takes over the earlier
    allocations (growing them when the new one is larger) and holds exactly
    the new data; an upload rejected for its arguments leaves the earlier
    channel as it was."""
    res, bsx = 128, 16
    gpu_ctx.set_topology(res, res, res, bsx)
    for n_spheres, seed in ((2, 1), (12, 2), (1, 3)):  # small, larger, smaller
        kind, vals = msbg_gpu.sphere_sdf_scene(res, bsx, n_spheres=n_spheres, rmin=6, rmax=24,
                                               seed=seed)
        upd = np.nonzero(kind == 1)[0].astype(np.int32)
        gpu_ctx.upload_channel(3, 0, kind, vals, 4.0, -4.0)
        assert np.array_equal(gpu_ctx.download_channel(3, np.empty_like(vals)), vals)
        gpu_ctx.apply_channel_pde_mcf(3, upd, 2, 0.1)
        got = gpu_ctx.download_channel(3, np.empty_like(vals))
        ref = oracle.mcf_oracle((res // bsx,) * 3, bsx, kind, vals, upd, 2, 0.1)
        ok, err = tol_ok(got, ref)
        assert ok, err
    bad = np.full(len(kind), 9, np.int8)
    with pytest.raises(msbg_gpu.MsbgError):
        gpu_ctx.upload_channel(3, 0, bad, vals, 4.0, -4.0)
    assert np.array_equal(gpu_ctx.download_channel(3, np.empty_like(got)), got)
