"""GPU MGPCG pressure solve (through the C ABI) against the FP64 oracle."""
import numpy as np
import pytest

import msbg_gpu
import oracle

pytestmark = pytest.mark.gpu


def rel_err(x, xo):
    return float(np.linalg.norm(x - xo) / max(1e-300, np.linalg.norm(xo)))


@pytest.mark.parametrize("res,bsx0,nl,band", [(64, 16, 2, 4.0), (128, 16, 2, 8.0),
                                              (128, 16, 3, 4.0), (128, 32, 2, 8.0)])
def test_mgpcg_converges_to_oracle(gpu_ctx, res, bsx0, nl, band):
    s = msbg_gpu.PressureScene(res, bsx0, nl, band=band, seed=11)
    gpu_ctx.pressure_prepare(s)
    info = gpu_ctx.pressure_solve(tol=1e-6)
    assert info.status == 0, info.status
    # recursive residual reached 1e-6; the true residual recomputed with the FP32
    # operator carries FP32 rounding (about 1e-5 at these sizes)
    assert info.relResidual <= 3e-5, info.relResidual
    assert info.iterations < 60
    x = gpu_ctx.pressure_download()
    b = gpu_ctx.pressure_download(rhs=True)
    xo, bo, it, rr = oracle.pressure_oracle(s, tol=1e-12)
    # same right-hand side (FP32 vs FP64 sampling)
    assert np.abs(b - bo).max() <= 1e-6 * np.abs(bo).max()
    # solution error against the FP64 oracle, FP32 solve to relative residual 1e-6
    assert rel_err(x, xo) <= 1e-5, rel_err(x, xo)


def test_mgpcg_graph_and_eager_agree(gpu_ctx):
    s = msbg_gpu.PressureScene(64, 16, 2, band=4.0, seed=4)
    gpu_ctx.pressure_prepare(s)
    a = gpu_ctx.pressure_solve(tol=1e-6, useGraph=1)
    xa = gpu_ctx.pressure_download()
    b = gpu_ctx.pressure_solve(tol=1e-6, useGraph=0)
    xb = gpu_ctx.pressure_download()
    assert a.iterations == b.iterations
    np.testing.assert_array_equal(xa, xb)


def test_mgpcg_is_deterministic(gpu_ctx):
    s = msbg_gpu.PressureScene(64, 16, 2, band=4.0, seed=6)
    gpu_ctx.pressure_prepare(s)
    gpu_ctx.pressure_solve(tol=1e-6)
    xa = gpu_ctx.pressure_download()
    gpu_ctx.pressure_solve(tol=1e-6)
    xb = gpu_ctx.pressure_download()
    np.testing.assert_array_equal(xa, xb)


def test_solve_without_prepare_is_an_error():
    ctx = msbg_gpu.Context(0)
    with pytest.raises(msbg_gpu.MsbgError):
        ctx.pressure_solve(tol=1e-6)
    ctx.close()


@pytest.mark.parametrize("res,bsx0,nl,band", [(128, 16, 2, 8.0), (128, 32, 2, 8.0),
                                              (128, 16, 3, 4.0)])
def test_fp64_refinement_reaches_true_residual_and_oracle(gpu_ctx, res, bsx0, nl, band):
    """Outer FP64 refinement: true residual <= 1e-6, error vs FP64 oracle <= 1e-5."""
    s = msbg_gpu.PressureScene(res, bsx0, nl, band=band, seed=11)
    gpu_ctx.pressure_prepare(s)
    info = gpu_ctx.pressure_solve(tol=1e-6, maxRefine=4)
    assert info.status == 0
    assert info.relResidual <= 1e-6, info.relResidual
    assert info.refinements >= 1
    xo, bo, it, rr = oracle.pressure_oracle(s, tol=1e-12)
    x64 = gpu_ctx.pressure_download(fp64=True)
    x32 = gpu_ctx.pressure_download()
    assert rel_err(x64, xo) <= 1e-5, rel_err(x64, xo)
    assert rel_err(x32, xo) <= 1e-5, rel_err(x32, xo)
    # the FP64 iterate's residual, recomputed by the oracle's own matrix
    r = bo - oracle.pressure_apply_oracle(s, x64)
    assert np.linalg.norm(r) <= 1.5e-6 * np.linalg.norm(bo)


@pytest.mark.parametrize("storage", [msbg_gpu.F16, msbg_gpu.BF16])
@pytest.mark.parametrize("res,bsx0,nl,band", [(128, 16, 2, 8.0), (128, 32, 2, 8.0),
                                              (128, 16, 3, 4.0)])
def test_16bit_vectors_under_fp64_refinement_reach_oracle(gpu_ctx, storage, res, bsx0, nl, band):
    """FP16 / BF16 level-0 vectors, FP32 arithmetic, FP64 refinement: the same
    true residual (1e-6) and the same distance to the FP64 oracle (1e-5) as the
    FP32 solve; the inner solves stop near the 16-bit rounding level, so more
    refinement steps are taken."""
    s = msbg_gpu.PressureScene(res, bsx0, nl, band=band, seed=11)
    gpu_ctx.pressure_prepare(s)
    ref = gpu_ctx.pressure_solve(tol=1e-6, maxRefine=4)
    assert ref.status == 0, ref.status
    info = gpu_ctx.pressure_solve(tol=1e-6, storage=storage, maxRefine=30)
    assert info.status == 0, info.status
    assert info.relResidual <= 1e-6, info.relResidual
    assert info.refinements >= 2
    assert info.iterations <= 4 * ref.iterations + 10, (info.iterations, ref.iterations)
    xo, bo, it, rr = oracle.pressure_oracle(s, tol=1e-12)
    x64 = gpu_ctx.pressure_download(fp64=True)
    assert rel_err(x64, xo) <= 1e-5, rel_err(x64, xo)
    r = bo - oracle.pressure_apply_oracle(s, x64)
    assert np.linalg.norm(r) <= 1.5e-6 * np.linalg.norm(bo)


def test_16bit_vectors_always_refine(gpu_ctx):
    """maxRefine = 0 with 16-bit storage still runs the FP64 refinement."""
    s = msbg_gpu.PressureScene(64, 16, 2, band=4.0, seed=3)
    gpu_ctx.pressure_prepare(s)
    info = gpu_ctx.pressure_solve(tol=1e-6, storage=msbg_gpu.F16, maxRefine=0)
    assert info.status == 0 and info.refinements >= 1
    assert info.relResidual <= 1e-6


def test_16bit_solves_are_deterministic(gpu_ctx):
    s = msbg_gpu.PressureScene(64, 16, 2, band=4.0, seed=8)
    gpu_ctx.pressure_prepare(s)
    out = []
    for _ in range(2):
        gpu_ctx.pressure_solve(tol=1e-6, storage=msbg_gpu.BF16, maxRefine=30)
        out.append(gpu_ctx.pressure_download(fp64=True))
    np.testing.assert_array_equal(out[0], out[1])


def test_unsupported_storage_is_rejected(gpu_ctx):
    s = msbg_gpu.PressureScene(64, 16, 2, band=4.0, seed=3)
    gpu_ctx.pressure_prepare(s)
    with pytest.raises(msbg_gpu.MsbgError):
        gpu_ctx.pressure_solve(tol=1e-6, storage=msbg_gpu.F64)


def test_uncovered_coarse_cells_read_as_zero():
    """Coarse cells under finer tiles that do not exist are never written by
    the restriction.  Here the context first fills and frees block tables of a
    smoother channel, so the pressure buffers allocated next start on recycled
    memory; the solve must still converge (it did not while those cells were
    left uninitialised and the recycled bits happened to be NaN patterns)."""
    ctx = msbg_gpu.Context(0)
    for _ in range(3):
        kind, vals = msbg_gpu.sphere_sdf_scene(256, 8, n_spheres=4, rmin=8, rmax=16, seed=5)
        ctx.set_topology(256, 256, 256, 8)
        ctx.upload_channel(1, 0, kind, vals[: int((kind == 1).sum())], 4.0, -4.0)
    ctx.set_topology(64, 64, 64, 8)  # frees the channel above
    s = msbg_gpu.PressureScene(128, 16, 2, band=8.0, seed=11)
    ctx.pressure_prepare(s)
    for storage in (msbg_gpu.F32, msbg_gpu.F16):
        info = ctx.pressure_solve(tol=1e-6, storage=storage, maxRefine=30)
        assert info.status == 0, (storage, info.status)
        assert info.relResidual <= 1e-6
    ctx.close()


@pytest.mark.parametrize("bsx0,nl,band", [(16, 2, 8.0), (32, 2, 8.0), (16, 3, 4.0)])
def test_pipelined_smoother_matches_per_tile_kernel(gpu_ctx, bsx0, nl, band):
    """Two level-0 smoothing sweeps (3 inner red-black iterations per tile)
    from x = 0: the persistent pipelined 16^3 kernel against the plain
    one-CTA-per-tile kernel, up to FP32 rounding of the sums."""
    s = msbg_gpu.PressureScene(128, bsx0, nl, band=band, seed=21)
    xs = []
    for what in (3, 0):  # 3: per-tile kernel, 0: pipelined kernel
        gpu_ctx.pressure_prepare(s)
        gpu_ctx.pressure_profile(what, 1, 3)
        xs.append(gpu_ctx.pressure_download())
    a, b = xs
    assert np.abs(a).max() > 0
    assert np.abs(a - b).max() <= 1e-5 * np.abs(a).max(), np.abs(a - b).max()


@pytest.mark.parametrize("bsx0,nl", [(32, 2), (16, 3)])
def test_packed_faces_change_no_bit(bsx0, nl, monkeypatch):
    """The V-cycle's packed x faces (the x-face halo read from contiguous
    copies of the neighbours' x = 0 / x = 15 planes) give the same solve, bit
    for bit, as the strided halo reads: same iterations, same pressure."""
    s = msbg_gpu.PressureScene(128, bsx0, nl, band=8.0, seed=31)
    out = []
    for faces in ("1", "0"):
        monkeypatch.setenv("MSBG_PRESSURE_FACES", faces)
        ctx = msbg_gpu.Context(0)
        try:
            ctx.pressure_prepare(s)
            res = []
            for storage in (msbg_gpu.F32, msbg_gpu.F16):
                info = ctx.pressure_solve(tol=1e-6, storage=storage, maxRefine=30)
                res.append((info.iterations, info.status, ctx.pressure_download()))
            out.append(res)
        finally:
            ctx.close()
    for (ia, sa, pa), (ib, sb, pb) in zip(*out):
        assert sa == 0 and sb == 0 and ia == ib
        assert np.array_equal(pa, pb)
