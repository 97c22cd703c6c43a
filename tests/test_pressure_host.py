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


def _host_apply(scene, x, dbc):
    L = msbg_gpu.lib()
    msbg_gpu._pressure_sigs(L)
    bl = np.ascontiguousarray(scene.block_levels, np.int32)
    d = None if dbc is None else np.array(dbc, np.int32)
    topo = msbg_gpu.TopoDesc(scene.res, scene.res, scene.res, scene.bsx0, scene.n_levels,
                             bl.ctypes.data_as(C.POINTER(C.c_int)),
                             None if d is None else d.ctypes.data_as(C.POINTER(C.c_int)))
    cb = scene.callbacks()
    y = np.zeros(len(x), np.float64)
    nm = C.c_int()
    fluid = np.zeros(32, np.int64)
    rc = L.msbg_gpu_pressure_host_check(C.byref(topo), C.byref(cb),
                                        x.ctypes.data_as(C.POINTER(C.c_float)),
                                        y.ctypes.data_as(C.POINTER(C.c_double)), C.byref(nm),
                                        fluid.ctypes.data_as(C.POINTER(C.c_int64)), None)
    return rc, y


def test_domain_boundary_spec_sets_the_wall_faces():
    """msbg_topo_desc.domainBc (setDomainBoundarySpec_, src/msbg.cpp:2462):
    p = 0 outside the grid, behind a coupling of 0 (DBC_SOLID), of the
    callback's coefficient on a lower face and 1 on an upper face (DBC_OPEN,
    the reference's constFaceCoeffAirBlock, src/msbg3.cpp:733-740), and with
    no spec the reference's own operator: lower faces as open, upper faces 0
    (computeDiagonalFLIP_, src/msbg3.cpp:2714-2722).  For x = 1, A x is the
    sum of the couplings to the outside and to air, so each rule shows as a
    constant on the liquid cells of one domain face."""
    from refgrid import OpenPool, to_blocks


    s = OpenPool()
    res = s.res
    x = np.ones(res ** 3, np.float32)
    zz, yy, xx = np.meshgrid(np.arange(res), np.arange(res), np.arange(res), indexing="ij")
    liq = zz < 12
    # couplings to air: the cells below the surface
    air = np.where(liq & (zz == 11), 0.5, 0.0)

    def expect(lo, hi):
        """lo/hi: coupling through each lower/upper domain face (x, y, z)"""
        e = air.copy()
        for ax, c in enumerate((xx, yy, zz)):
            e += np.where(liq & (c == 0), lo[ax], 0.0)
            e += np.where(liq & (c == res - 1), hi[ax], 0.0)
        return to_blocks(np.where(liq, e, 0.0), s.bsx0)

    cases = [([1] * 6, (0, 0, 0), (0, 0, 0)),
             ([0] * 6, (0.5, 0.5, 0.5), (1, 1, 1)),
             ([1, 0, 0, 1, 1, 1], (0, 0.5, 0), (1, 0, 0)),
             (None, (0.5, 0.5, 0.5), (0, 0, 0))]
    for dbc, lo, hi in cases:
        rc, y = _host_apply(s, x, dbc)
        assert rc == 0
        assert np.allclose(y, expect(lo, hi)), dbc
        yo = oracle.pressure_apply_oracle(s, x.astype(np.float64), domain_bc=dbc)
        assert np.abs(y - yo).max() <= 1e-6, dbc
    bad = [0, 1, 1, 1, 1, 2]  # not a DBC_* value
    assert _host_apply(s, x, bad)[0] == 5


@pytest.mark.parametrize("res,bsx0,nl,band", SCENES)
def test_array_build_equals_callback_build(res, bsx0, nl, band):
    """The bulk prepare's arrays (msbg_scene_pressure_arrays samples each cell
    at its lowest fine voxel, as the callbacks are asked) build the callback
    build's level-0 operator: bit-identical where no face reads a coarser
    block at another fine voxel of its cell, and the same liquid cells on
    every level."""
    from refgrid import interface_mask

    s = msbg_gpu.PressureScene(res, bsx0, nl, band=band, seed=5)
    flags, face, rhs = s.arrays()
    x = np.random.default_rng(2).standard_normal(s.packed_size()).astype(np.float32)
    y_cb, nm_cb, fl_cb, _ = host_check(s, x)
    L = msbg_gpu.lib()
    fn = L.msbg_gpu_pressure_host_check_arrays
    fn.restype = C.c_int
    bl = np.ascontiguousarray(s.block_levels, np.int32)
    d = msbg_gpu.TopoDesc(res, res, res, bsx0, nl, bl.ctypes.data_as(C.POINTER(C.c_int)))
    P = lambda a, t: a.ctypes.data_as(C.POINTER(t))
    y = np.zeros(len(x))
    nm = C.c_int()
    fluid = np.zeros(32, np.int64)
    rc = fn(C.byref(d), P(flags, C.c_uint16), P(face[0], C.c_float), P(face[1], C.c_float),
            P(face[2], C.c_float), P(rhs, C.c_float), P(x, C.c_float), P(y, C.c_double),
            C.byref(nm), P(fluid, C.c_int64), None)
    assert rc == 0
    assert nm.value == nm_cb and (fluid[:nm.value] == fl_cb).all()
    iface = interface_mask(s.block_levels, res, bsx0)
    assert np.array_equal(y[~iface], y_cb[~iface])
    assert np.abs(y - y_cb).max() <= 1e-6 * np.abs(y_cb).max()


def test_galerkin_levels_of_a_three_level_grid_are_exact():
    """A tile of a uniform coarse level spans several blocks, some of whose
    cells aggregate at that level and some not (a 3-level grid around a wavy
    surface): every coarse level is still P^T A P on every cell."""
    s = msbg_gpu.PressureScene(512, 32, 3, z_liquid=0.3, n_spheres=32, r_min=20 / 4096,
                               r_max=60 / 4096, n_cuboids=0, band=(48.0 - 16 * 3 ** 0.5) / 8,
                               seed=4096, wave_amp=0.05, n_waves=8)
    x = np.zeros(s.packed_size(), np.float32)
    _, nmg, _, gerr = host_check(s, x)
    assert nmg >= 5
    assert gerr.max() < 1e-6, gerr
