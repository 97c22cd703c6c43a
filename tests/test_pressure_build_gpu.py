"""The bulk prepare builds the hierarchy's per-cell arrays on the GPU
(build_gpu.cu); the host build (MSBG_PRESSURE_BUILD=host) of the same arrays is
its reference:
  - MG level 0: the same expressions in the same order, so the diagonal and
    the right-hand side are bit-identical and A x agrees to FP32 rounding of
    the product;
  - the Galerkin levels: exact sums over the liquid children in another
    order, so A_c x agrees to 1e-6 of max |A_c x| (checked on the levels in
    block layout; the uniform levels below enter through the solve);
  - the solves agree to the solver tolerance, and unsolvable input is
    reported the same way."""
import os

import numpy as np
import pytest

import msbg_gpu

pytestmark = pytest.mark.gpu

CASES = [(128, 32, 2, 16.0, None), (128, 16, 3, 8.0, None), (64, 8, 2, 4.0, None),
         (128, 32, 2, 16.0, [1, 1, 1, 0, 1, 1])]


def prepared(ctx, scene, arrays, host, dbc=None):
    os.environ["MSBG_PRESSURE_BUILD"] = "host" if host else "device"
    try:
        flags, face, rhs = arrays
        ctx.pressure_prepare_arrays(scene.res, scene.bsx0, scene.n_levels, scene.block_levels,
                                    flags, face, rhs, domain_bc=dbc)
    finally:
        os.environ.pop("MSBG_PRESSURE_BUILD", None)


def level_count(ctx):
    import ctypes as C
    st = msbg_gpu.PressureStats()
    L = msbg_gpu.lib()
    ctx._check(L.msbg_gpu_pressure_stats(ctx._h, C.byref(st)), "stats")
    return st.nMgLevels, [int(st.fluid[m]) for m in range(st.nMgLevels)]


@pytest.mark.parametrize("res,bsx0,nl,band,dbc", CASES)
def test_device_build_equals_host_build(res, bsx0, nl, band, dbc):
    scene = msbg_gpu.PressureScene(res, bsx0, nl, band=band, seed=9)
    arrays = scene.arrays()
    out = {}
    for host in (True, False):
        ctx = msbg_gpu.Context(0)
        try:
            prepared(ctx, scene, arrays, host, dbc)
            nmg, fluid = level_count(ctx)
            diag0 = ctx.diagonal(0)
            rhs = ctx.pressure_download(rhs=True)
            ys = []
            # the levels the component entry points address in block layout
            for m in range(min(nmg - 1, scene.n_levels)):
                rng = np.random.default_rng(100 + m)  # the same x on both sides
                x = rng.standard_normal(ctx.level_size(m)).astype(np.float32)
                ys.append((x, ctx.matvec(m, x)))
            info = ctx.pressure_solve(tol=1e-6, maxRefine=30)
            p = ctx.pressure_download(fp64=True)
            out[host] = (nmg, fluid, diag0, rhs, ys, info.status, p)
        finally:
            ctx.close()
    h, d = out[True], out[False]
    assert h[0] == d[0] and h[1] == d[1]
    assert np.array_equal(h[2], d[2])
    assert np.array_equal(h[3], d[3])
    for m, ((xh, yh), (xd, yd)) in enumerate(zip(h[4], d[4])):
        assert np.array_equal(xh, xd)
        tol = 1e-6 * np.abs(yh).max()
        assert np.abs(yh - yd).max() <= tol, m
    assert h[5] == 0 and d[5] == 0
    assert np.linalg.norm(h[6] - d[6]) <= 1e-5 * np.linalg.norm(h[6])


def test_device_build_reports_an_isolated_liquid_cell():
    from refgrid import box_problem

    flags, face, rhs = box_problem(res=32, bsx0=16, z_liquid=20, seed=1)
    # a liquid cell whose six faces have coefficient 0, with b != 0
    c = 5 + 16 * 5 + 256 * 5  # cell (5, 5, 5) of block 0
    for f in face:
        f[c] = 0.0
    face[0][c + 1] = 0.0
    face[1][c + 16] = 0.0
    face[2][c + 256] = 0.0
    rhs[c] = 1.0
    ctx = msbg_gpu.Context(0)
    try:
        with pytest.raises(msbg_gpu.MsbgError) as e:
            ctx.pressure_prepare_arrays(32, 16, 2, np.zeros(8, np.int32), flags, face, rhs)
        assert "(5,5,5)" in str(e.value)
        rhs[c] = 0.0  # consistent: dropped, and the rest solves
        ctx.pressure_prepare_arrays(32, 16, 2, np.zeros(8, np.int32), flags, face, rhs)
        assert ctx.pressure_solve(tol=1e-6, maxRefine=30).status == 0
    finally:
        ctx.close()


@pytest.mark.parametrize("res,bsx0,nl,band,dbc", CASES[:2] + CASES[3:])
def test_pinned_arrays_build_the_same_bits(res, bsx0, nl, band, dbc):
    """The caller's arrays in page-locked host memory (the e2e bench keeps
    them there) give the same operator and solve as pageable ones, bit for
    bit, and a pinned output buffer receives the same pressure."""
    scene = msbg_gpu.PressureScene(res, bsx0, nl, band=band, seed=9)
    out = []
    for pinned in (False, True):
        arrays = scene.arrays(pinned=pinned)
        ctx = msbg_gpu.Context(0)
        try:
            prepared(ctx, scene, arrays, False, dbc)
            info = ctx.pressure_solve(tol=1e-6, maxRefine=30)
            p = (msbg_gpu.pinned_empty(ctx.pressure_download().shape, np.float32)
                 if pinned else None)
            out.append((level_count(ctx), ctx.diagonal(0), ctx.pressure_download(rhs=True),
                        info.iterations, ctx.pressure_download(fp64=True),
                        ctx.pressure_download(out=p)))
        finally:
            ctx.close()
    a, b = out
    assert a[0] == b[0] and a[3] == b[3]
    for u, v in zip(a[1:3] + a[4:], b[1:3] + b[4:]):
        assert np.array_equal(u, v)
