"""CPU tests of the pressure hierarchy: operator vs the FP64 oracle, Galerkin."""
import ctypes as C

import numpy as np
import pytest

import msbg_gpu
import oracle


def host_check(scene, x):
    L = msbg_gpu.lib()
    msbg_gpu._pressure_sigs(L)
    fn = L.msbg_gpu_pressure_host_check
    fn.restype = C.c_int
    fn.argtypes = [C.POINTER(msbg_gpu.TopoDesc), C.POINTER(msbg_gpu.PressureCallbacks),
                   C.POINTER(C.c_float), C.POINTER(C.c_double), C.POINTER(C.c_int),
                   C.POINTER(C.c_int64), C.POINTER(C.c_double)]
    bl = np.ascontiguousarray(scene.block_levels, np.int32)
    d = msbg_gpu.TopoDesc(scene.res, scene.res, scene.res, scene.bsx0, scene.n_levels,
                          bl.ctypes.data_as(C.POINTER(C.c_int)))
    cb = scene.callbacks()
    x = np.ascontiguousarray(x, np.float32)
    y = np.zeros(len(x))
    nm = C.c_int()
    fluid = np.zeros(32, np.int64)
    gerr = np.zeros(32)
    rc = fn(C.byref(d), C.byref(cb), x.ctypes.data_as(C.POINTER(C.c_float)),
            y.ctypes.data_as(C.POINTER(C.c_double)), C.byref(nm),
            fluid.ctypes.data_as(C.POINTER(C.c_int64)), gerr.ctypes.data_as(C.POINTER(C.c_double)))
    assert rc == 0
    return y, nm.value, fluid[:nm.value], gerr[:nm.value - 1]


SCENES = [(64, 16, 2, 4.0), (128, 16, 2, 8.0), (128, 16, 3, 4.0), (64, 8, 3, 2.0)]


@pytest.mark.parametrize("res,bsx0,nl,band", SCENES)
def test_level0_operator_matches_oracle_and_coarse_levels_are_galerkin(res, bsx0, nl, band):
    s = msbg_gpu.PressureScene(res, bsx0, nl, band=band, seed=5)
    assert len(np.unique(s.block_levels)) >= min(2, nl) or res == 64
    x = np.random.default_rng(1).standard_normal(s.packed_size()).astype(np.float32)
    y, nmg, fluid, gerr = host_check(s, x)
    yo = oracle.pressure_apply_oracle(s, x.astype(np.float64))
    assert np.abs(y - yo).max() <= 1e-6 * np.abs(yo).max()
    assert nmg >= 3
    assert fluid[-1] <= 512
    assert all(fluid[m + 1] <= fluid[m] for m in range(nmg - 1))
    assert gerr.max() < 1e-6


def test_adaptive_scene_has_two_levels_and_graded_map():
    s = msbg_gpu.PressureScene(128, 16, 2, band=8.0, seed=5)
    lv = s.block_levels.reshape(8, 8, 8)
    assert set(np.unique(lv)) == {0, 1}
    # 2:1 grading over face neighbours
    for ax in range(3):
        assert np.abs(np.diff(lv, axis=ax)).max() <= 1


def test_oracle_solution_satisfies_system():
    s = msbg_gpu.PressureScene(64, 16, 2, band=4.0, seed=3)
    x, b, it, rr = oracle.pressure_oracle(s, tol=1e-12)
    assert rr < 1e-11
    ax = oracle.pressure_apply_oracle(s, x)
    assert np.abs(ax - b).max() <= 1e-9 * np.abs(b).max()


def test_domain_boundary_spec_sets_the_wall_faces():
    """msbg_topo_desc.domainBc: a DBC_SOLID domain face has no coupling, a
    DBC_OPEN one couples to p = 0 outside with the callback's coefficient
    (setDomainBoundarySpec_, src/msbg.cpp:2462).  A pool (liquid below z = 12,
    air above) whose face callback returns 1 everywhere, walls solid: opening
    the -x face adds one coupling to each liquid cell at x = 0, so A x for
    x = 1 differs by exactly 1 there and nowhere else."""
    import ctypes as C

    import numpy as np

    import msbg_gpu
    from refgrid import to_blocks

    res, bsx0 = 16, 16
    L = msbg_gpu.lib()
    msbg_gpu._pressure_sigs(L)
    ct = C.CFUNCTYPE(C.c_uint16, C.c_void_p, C.c_int, C.c_int, C.c_int)(
        lambda u, x, y, z: 0 if z < 12 else 0x1000)
    fc = C.CFUNCTYPE(C.c_float, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int)(
        lambda u, d, x, y, z: 1.0)
    rh = C.CFUNCTYPE(C.c_float, C.c_void_p, C.c_int, C.c_int, C.c_int)(lambda u, x, y, z: 1.0)
    cb = msbg_gpu.PressureCallbacks(C.cast(ct, C.c_void_p).value, C.cast(fc, C.c_void_p).value,
                                    C.cast(rh, C.c_void_p).value, None)
    bl = np.zeros(1, np.int32)
    x = np.ones(res ** 3, np.float32)
    ys = []
    for dbc in ([1, 1, 1, 1, 1, 1], [0, 1, 1, 1, 1, 1]):
        d = np.array(dbc, np.int32)
        topo = msbg_gpu.TopoDesc(res, res, res, bsx0, 2, bl.ctypes.data_as(C.POINTER(C.c_int)),
                                 d.ctypes.data_as(C.POINTER(C.c_int)))
        y = np.zeros(res ** 3, np.float64)
        nm = C.c_int()
        fluid = np.zeros(32, np.int64)
        rc = L.msbg_gpu_pressure_host_check(C.byref(topo), C.byref(cb),
                                            x.ctypes.data_as(C.POINTER(C.c_float)),
                                            y.ctypes.data_as(C.POINTER(C.c_double)), C.byref(nm),
                                            fluid.ctypes.data_as(C.POINTER(C.c_int64)), None)
        assert rc == 0
        ys.append(y)
    zz, yy, xx = np.meshgrid(np.arange(res), np.arange(res), np.arange(res), indexing="ij")
    face = to_blocks(((xx == 0) & (zz < 12)).astype(np.float32), bsx0) > 0
    diff = ys[1] - ys[0]
    assert np.allclose(diff[face], 1.0) and np.allclose(diff[~face], 0.0)
    bad = np.array([0, 1, 1, 1, 1, 2], np.int32)  # not a DBC_* value
    topo = msbg_gpu.TopoDesc(res, res, res, bsx0, 2, bl.ctypes.data_as(C.POINTER(C.c_int)),
                             bad.ctypes.data_as(C.POINTER(C.c_int)))
    nm = C.c_int()
    assert L.msbg_gpu_pressure_host_check(C.byref(topo), C.byref(cb), None, None, C.byref(nm),
                                          None, None) == 5
