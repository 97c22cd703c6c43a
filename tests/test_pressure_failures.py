"""Solver failures made on the host, with no GPU fault: the status and error
codes a caller sees (the reference reports these through its PCG's return
path, src/msbg3.cpp:3168-3171 and 3217-3219, and exits on its asserts; this
library returns codes instead).

  - a non-finite right-hand side: the solve ends with status 3 (non-finite);
  - maxIter reached before the tolerance: status 1;
  - a liquid cell coupled to nothing (all six face coefficients 0) with a
    nonzero right-hand side: no pressure satisfies its equation, and the
    prepare fails with MSBG_EMATH; with a zero right-hand side the cell is
    dropped (p = 0) and the solve proceeds;
  - a non-finite face coefficient of a liquid cell: MSBG_EMATH at prepare.
The prepare-time checks run in the host build, so they are tested on CPU
through msbg_gpu_pressure_host_check as well as on the GPU.
"""
import ctypes as C

import numpy as np
import pytest

import msbg_gpu
from refgrid import box_problem

RES, BSX0, NL = 32, 16, 2
MSBG_EMATH = 15


def _isolate(flags, face, rhs, cell=(8, 8, 8), value=1.0):
    """Zero the six faces of one liquid cell (x, y, z) and set its rhs."""
    from refgrid import to_blocks

    dense = [np.zeros((RES,) * 3, np.float32) for _ in range(3)]
    x, y, z = cell
    for d in range(3):
        m = np.zeros((RES,) * 3, bool)
        m[z, y, x] = True                       # the cell's own lower face
        up = [z, y, x]
        up[2 - d] += 1
        m[tuple(up)] = True                     # the +1 neighbour's lower face
        face[d] = np.where(to_blocks(m, BSX0), 0.0, face[d]).astype(np.float32)
    r = np.zeros((RES,) * 3, np.float32)
    r[z, y, x] = 1.0
    sel = to_blocks(r, BSX0) > 0
    rhs = rhs.copy()
    rhs[sel] = value
    return flags, face, rhs


def _host_check(flags, face, rhs):
    """Runs the host build of the hierarchy through msbg_gpu_pressure_host_check
    with callbacks over the arrays; returns (rc, liquid cells of MG level 0)."""
    import oracle

    A = oracle.ArrayScene(RES, BSX0, NL, np.zeros((RES // BSX0) ** 3, np.int32), flags, face, rhs)
    L = msbg_gpu.lib()
    msbg_gpu._pressure_sigs(L)
    cb = A.callbacks()
    pcb = msbg_gpu.PressureCallbacks(cb.sampleCellType, cb.sampleFaceCoeff, cb.sampleRhs, cb.user)
    bl = np.zeros((RES // BSX0) ** 3, np.int32)
    d = msbg_gpu.TopoDesc(RES, RES, RES, BSX0, NL, bl.ctypes.data_as(C.POINTER(C.c_int)))
    nm = C.c_int()
    fluid = np.zeros(32, np.int64)
    rc = L.msbg_gpu_pressure_host_check(C.byref(d), C.byref(pcb), None, None, C.byref(nm),
                                        fluid.ctypes.data_as(C.POINTER(C.c_int64)), None)
    A.close()
    return rc, int(fluid[0])


def test_isolated_cell_with_rhs_is_a_math_error_on_host():
    flags, face, rhs = box_problem(RES, BSX0)
    rc0, n0 = _host_check(flags, face, rhs)
    assert rc0 == 0
    rc, _ = _host_check(*_isolate(flags, list(face), rhs, value=1.0))
    assert rc == MSBG_EMATH
    rc, n = _host_check(*_isolate(flags, list(face), rhs, value=0.0))
    assert rc == 0 and n == n0 - 1


def test_non_finite_face_coefficient_is_a_math_error_on_host():
    flags, face, rhs = box_problem(RES, BSX0)
    face = list(face)
    face[1] = face[1].copy()
    face[1][np.nonzero(flags == 0)[0][100]] = np.inf
    rc, _ = _host_check(flags, face, rhs)
    assert rc == MSBG_EMATH


def _ctx(flags, face, rhs):
    ctx = msbg_gpu.Context(0)
    ctx.pressure_prepare_arrays(RES, BSX0, NL, np.zeros((RES // BSX0) ** 3, np.int32), flags,
                                face, rhs)
    return ctx


@pytest.mark.gpu
@pytest.mark.parametrize("bad", [np.nan, np.inf])
@pytest.mark.parametrize("max_refine", [0, 4])
def test_non_finite_rhs_gives_status_3(bad, max_refine):
    flags, face, rhs = box_problem(RES, BSX0)
    rhs = rhs.copy()
    rhs[np.nonzero(flags == 0)[0][1234]] = bad
    ctx = _ctx(flags, face, rhs)
    try:
        info = ctx.pressure_solve(tol=1e-6, maxRefine=max_refine)
        assert info.status == 3
    finally:
        ctx.close()


@pytest.mark.gpu
@pytest.mark.parametrize("max_refine", [0, 4])
def test_max_iter_gives_status_1(max_refine):
    flags, face, rhs = box_problem(RES, BSX0)
    ctx = _ctx(flags, face, rhs)
    try:
        info = ctx.pressure_solve(tol=1e-12, maxIter=1, maxRefine=max_refine)
        assert info.status == 1
        ok = ctx.pressure_solve(tol=1e-6, maxRefine=max_refine)
        assert ok.status == 0  # the context stays usable
    finally:
        ctx.close()


@pytest.mark.gpu
def test_isolated_cell_with_rhs_fails_the_prepare():
    flags, face, rhs = box_problem(RES, BSX0)
    with pytest.raises(msbg_gpu.MsbgError) as ei:
        _ctx(*_isolate(flags, list(face), rhs, value=1.0))
    assert ei.value.code == MSBG_EMATH
    ctx = _ctx(*_isolate(flags, list(face), rhs, value=0.0))
    try:
        assert ctx.pressure_solve(tol=1e-6, maxRefine=4).status == 0
    finally:
        ctx.close()
