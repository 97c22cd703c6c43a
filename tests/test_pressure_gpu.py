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
