"""Python binding (ctypes) of the C ABI in include/msbg_gpu.h.

Thin: every call goes straight to libmsbg_gpu.so (the sm_100a kernels); there
is no Python or CPU compute path.  If the library is missing the import of
:func:`lib` raises, so nothing can silently fall back.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.dirname(HERE)
LIB_PATH = os.path.join(PKG, "libmsbg_gpu.so")
SCENE_LIB_PATH = os.path.join(PKG, "libmsbg_scene.so")

MSBG_OK = 0
STATUS = {0: "MSBG_OK", 1: "MSBG_ERROR", 2: "MSBG_ENOMEM", 4: "MSBG_ENOTIMPL",
          5: "MSBG_EINVARG", 15: "MSBG_EMATH", 20: "MSBG_EINTERNAL", 25: "MSBG_ENODEV",
          30: "MSBG_ETIMEOUT"}

BLOCK_NULL, BLOCK_VALUE, BLOCK_EMPTY, BLOCK_FULL = 0, 1, 2, 3

# storage types of the solver vectors (msbg_gpu_solve_params.storage)
F32, F16, BF16, F64 = 0, 1, 2, 3

_lib = None
_scene_lib = None


class MsbgError(RuntimeError):
    def __init__(self, code, msg=""):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code


class TopoDesc(C.Structure):
    _fields_ = [("sx", C.c_int), ("sy", C.c_int), ("sz", C.c_int), ("bsx0", C.c_int),
                ("nLevels", C.c_int), ("blockLevel", C.POINTER(C.c_int)),
                ("domainBc", C.POINTER(C.c_int))]

DBC_OPEN, DBC_SOLID = 0, 1


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


def lib():
    """Load libmsbg_gpu.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} missing: run msbg-flip_b200/build.py")
    L = C.CDLL(LIB_PATH)
    vp, i32, f32 = C.c_void_p, C.c_int, C.c_float
    pi32 = C.POINTER(C.c_int)
    pi8 = C.POINTER(C.c_int8)
    pf32 = C.POINTER(C.c_float)
    sig = {
        "msbg_gpu_init": (i32, [i32, C.POINTER(vp)]),
        "msbg_gpu_destroy": (i32, [vp]),
        "msbg_gpu_last_error": (C.c_char_p, [vp]),
        "msbg_gpu_sync": (i32, [vp]),
        "msbg_gpu_stream": (i32, [vp, C.POINTER(vp)]),
        "msbg_gpu_sync_topology": (i32, [vp, C.POINTER(TopoDesc)]),
        "msbg_gpu_upload_channel": (i32, [vp, i32, i32, pi8, C.POINTER(pf32), pf32, f32, f32]),
        "msbg_gpu_download_channel": (i32, [vp, i32, C.POINTER(pf32), pf32]),
        "msbg_gpu_upload_channel_u16": (i32, [vp, i32, i32, pi8, C.POINTER(C.POINTER(C.c_uint16)),
                                              C.POINTER(C.c_uint16), C.c_uint16, C.c_uint16]),
        "msbg_gpu_download_channel_u16": (i32, [vp, i32, C.POINTER(C.POINTER(C.c_uint16)),
                                                C.POINTER(C.c_uint16)]),
        "msbg_gpu_channel_num_value_blocks": (i32, [vp, i32, C.POINTER(C.c_int64)]),
        "msbg_gpu_channel_device_ptr": (i32, [vp, i32, C.POINTER(vp)]),
        "msbg_gpu_pde_mcf": (i32, [vp, i32, pi32, i32, i32, f32, i32]),
        "msbg_gpu_pde_mcf_device": (i32, [vp, vp, vp, vp, pi32, i32, i32, i32, i32, f32, f32,
                                          i32, f32, i32, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def scene_lib():
    """Load libmsbg_scene.so, the seeded input generators (include/msbg_scene.h).
    It is separate from the solver library and does not load it."""
    global _scene_lib
    if _scene_lib is not None:
        return _scene_lib
    if not os.path.exists(SCENE_LIB_PATH):
        raise ImportError(f"{SCENE_LIB_PATH} missing: run msbg-flip_b200/build.py")
    L = C.CDLL(SCENE_LIB_PATH)
    vp, i32, f32 = C.c_void_p, C.c_int, C.c_float
    sig = {
        "msbg_scene_sphere_sdf": (i32, [i32, i32, i32, f32, f32, f32, i32, C.c_uint64,
                                        C.POINTER(C.c_int8), C.POINTER(C.c_float),
                                        C.POINTER(C.c_int64)]),
        "msbg_scene_pressure_create": (vp, [i32, i32, i32, f32, i32, f32, f32, i32, i32, i32, f32,
                                            C.c_uint64]),
        "msbg_scene_pressure_create_wavy": (vp, [i32, i32, i32, f32, f32, i32, i32, f32, f32, i32,
                                                 i32, i32, f32, C.c_uint64]),
        "msbg_scene_pressure_destroy": (None, [vp]),
        "msbg_scene_pressure_block_levels": (i32, [vp, C.POINTER(C.c_int)]),
        "msbg_scene_pressure_arrays": (i32, [vp, C.POINTER(C.c_uint16)] +
                                       [C.POINTER(C.c_float)] * 4),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    _scene_lib = L
    return L


def sphere_sdf_scene(res, bsx, n_spheres=64, rmin=20.0, rmax=60.0, band=4.0, dilate=1,
                     seed=1234, with_values=True):
    """Seeded union-of-spheres signed distance field on a single-level grid.

    Returns (kind[nb] int8, values[nValue, bsx, bsx, bsx] float32 or None).
    """
    L = scene_lib()
    nb = (res // bsx) ** 3
    kind = np.zeros(nb, np.int8)
    nval = C.c_int64(0)
    rc = L.msbg_scene_sphere_sdf(res, bsx, n_spheres, rmin, rmax, band, dilate, seed,
                                 _p(kind, C.c_int8), None, C.byref(nval))
    if rc:
        raise MsbgError(rc, "scene generation")
    if not with_values:
        return kind, None
    vals = np.empty((nval.value, bsx, bsx, bsx), np.float32)
    rc = L.msbg_scene_sphere_sdf(res, bsx, n_spheres, rmin, rmax, band, dilate, seed,
                                 _p(kind, C.c_int8), _p(vals, C.c_float), C.byref(nval))
    if rc:
        raise MsbgError(rc, "scene generation")
    return kind, vals


class Context:
    """One device context (stream + device pools); mirrors the MSBG calls."""

    def __init__(self, device=0):
        L = lib()
        h = C.c_void_p()
        rc = L.msbg_gpu_init(device, C.byref(h))
        if rc:
            raise MsbgError(rc, "msbg_gpu_init")
        self._h = h
        self._L = L
        self.device = device

    def _check(self, rc, what):
        if rc != MSBG_OK:
            msg = self._L.msbg_gpu_last_error(self._h)
            raise MsbgError(rc, f"{what}: {msg.decode() if msg else ''}")

    def close(self):
        if self._h:
            self._L.msbg_gpu_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def sync(self):
        self._check(self._L.msbg_gpu_sync(self._h), "sync")

    def set_topology(self, sx, sy, sz, bsx0, n_levels=1, block_level=None):
        bl = None
        if block_level is not None:
            self._bl = np.ascontiguousarray(block_level, np.int32)
            bl = _p(self._bl, C.c_int)
        d = TopoDesc(sx, sy, sz, bsx0, n_levels, bl)
        self._check(self._L.msbg_gpu_sync_topology(self._h, C.byref(d)), "sync_topology")
        self.n_blocks = (sx // bsx0) * (sy // bsx0) * (sz // bsx0)
        self._bsx0 = bsx0
        self._levels = (np.array(self._bl) if block_level is not None
                        else np.zeros(self.n_blocks, np.int32))

    def upload_channel(self, chan, level, kind, packed, empty_val=0.0, full_val=0.0):
        kind = np.ascontiguousarray(kind, np.int8)
        packed = np.ascontiguousarray(packed, np.float32)
        self._check(self._L.msbg_gpu_upload_channel(
            self._h, chan, level, _p(kind, C.c_int8), None, _p(packed, C.c_float),
            empty_val, full_val), "upload_channel")
        self.sync()

    def upload_channel_blocks(self, chan, level, kind, blocks, empty_val=0.0, full_val=0.0):
        """Upload from per-block host arrays (blocks[bid] or None), as MSBG holds them."""
        kind = np.ascontiguousarray(kind, np.int8)
        ptrs = (C.POINTER(C.c_float) * len(kind))()
        keep = []
        for b, arr in enumerate(blocks):
            if arr is not None:
                a = np.ascontiguousarray(arr, np.float32)
                keep.append(a)
                ptrs[b] = _p(a, C.c_float)
        self._check(self._L.msbg_gpu_upload_channel(
            self._h, chan, level, _p(kind, C.c_int8), ptrs, None, empty_val, full_val),
            "upload_channel")
        self.sync()

    def download_channel(self, chan, out):
        self._check(self._L.msbg_gpu_download_channel(self._h, chan, None, _p(out, C.c_float)),
                    "download_channel")
        return out

    def upload_channel_u16(self, chan, level, kind, packed, empty_val=0, full_val=0):
        """msbg_gpu_upload_channel_u16: a 16-bit render-density channel (raw values)."""
        kind = np.ascontiguousarray(kind, np.int8)
        packed = np.ascontiguousarray(packed, np.uint16)
        self._check(self._L.msbg_gpu_upload_channel_u16(
            self._h, chan, level, _p(kind, C.c_int8), None, _p(packed, C.c_uint16),
            int(empty_val), int(full_val)), "upload_channel_u16")
        self.sync()

    def download_channel_u16(self, chan, out):
        self._check(self._L.msbg_gpu_download_channel_u16(self._h, chan, None,
                                                          _p(out, C.c_uint16)),
                    "download_channel_u16")
        return out

    def stream(self):
        """The context's CUDA stream handle (an int), e.g. for
        torch.cuda.ExternalStream."""
        p = C.c_void_p()
        self._check(self._L.msbg_gpu_stream(self._h, C.byref(p)), "stream")
        return p.value or 0

    def num_value_blocks(self, chan):
        n = C.c_int64()
        self._check(self._L.msbg_gpu_channel_num_value_blocks(self._h, chan, C.byref(n)), "nvb")
        return n.value

    def device_ptr(self, chan):
        p = C.c_void_p()
        self._check(self._L.msbg_gpu_channel_device_ptr(self._h, chan, C.byref(p)), "dptr")
        return p.value

    def apply_channel_pde_mcf(self, chan, block_list, num_iter, dt, clamp01=False, sync=True):
        """msbg_gpu_pde_mcf: replaces applyChannelPdeFast<float>(MCF, 8-colour)."""
        bl = np.ascontiguousarray(block_list, np.int32)
        self._check(self._L.msbg_gpu_pde_mcf(self._h, chan, _p(bl, C.c_int), len(bl),
                                             num_iter, dt, int(bool(clamp01))), "pde_mcf")
        if sync:
            self.sync()


# ---------------------------------------------------------------------------
# FLIP pressure solve
# ---------------------------------------------------------------------------
CELL_TYPE_FN = C.CFUNCTYPE(C.c_uint16, C.c_void_p, C.c_int, C.c_int, C.c_int)
FACE_FN = C.CFUNCTYPE(C.c_float, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int)
RHS_FN = C.CFUNCTYPE(C.c_float, C.c_void_p, C.c_int, C.c_int, C.c_int)


class PressureCallbacks(C.Structure):
    _fields_ = [("sampleCellType", C.c_void_p), ("sampleFaceCoeff", C.c_void_p),
                ("sampleRhs", C.c_void_p), ("user", C.c_void_p)]


class SolveParams(C.Structure):
    _fields_ = [("nPre", C.c_int), ("nPost", C.c_int), ("nCoarse", C.c_int),
                ("maxIter", C.c_int), ("tol", C.c_float), ("innerIter", C.c_int),
                ("storage", C.c_int), ("maxRefine", C.c_int), ("useGraph", C.c_int),
                ("coarseScale", C.c_float), ("learned", C.c_int)]


class SolveInfo(C.Structure):
    _fields_ = [("iterations", C.c_int), ("refinements", C.c_int), ("status", C.c_int),
                ("relResidual", C.c_double), ("solveSeconds", C.c_double),
                ("fineCells", C.c_int64), ("nMgLevels", C.c_int),
                ("kernelLaunches", C.c_int64), ("initialRelResidual", C.c_double),
                ("learnedFallback", C.c_int)]


class PressureStats(C.Structure):
    _fields_ = [("nMgLevels", C.c_int), ("coarseCells", C.c_int),
                ("cells", C.c_int64 * 32), ("fluid", C.c_int64 * 32), ("tiles", C.c_int64 * 32),
                ("h2dBytes", C.c_int64), ("deviceBytesUsed", C.c_int64),
                ("prepareSeconds", C.c_double), ("buildSeconds", C.c_double)]


def _pressure_sigs(L):
    vp, i32 = C.c_void_p, C.c_int
    sig = {
        "msbg_gpu_solve_params_default": (None, [C.POINTER(SolveParams)]),
        "msbg_gpu_pressure_prepare": (i32, [vp, C.POINTER(TopoDesc), C.POINTER(PressureCallbacks)]),
        "msbg_gpu_pressure_solve": (i32, [vp, C.POINTER(SolveParams), C.POINTER(SolveInfo)]),
        "msbg_gpu_pressure_download": (i32, [vp, C.POINTER(C.c_float), C.c_int64]),
        "msbg_gpu_pressure_download_rhs": (i32, [vp, C.POINTER(C.c_float), C.c_int64]),
        "msbg_gpu_pressure_download64": (i32, [vp, C.POINTER(C.c_double), C.c_int64]),
        "msbg_gpu_pressure_packed_size": (i32, [vp, C.POINTER(C.c_int64)]),
        "msbg_gpu_pressure_stats": (i32, [vp, C.POINTER(PressureStats)]),
        "msbg_gpu_pressure_profile": (i32, [vp, i32, i32, i32, C.POINTER(C.c_double),
                                            C.POINTER(C.c_double)]),
        "msbg_gpu_pressure_prepare_arrays": (i32, [vp, C.POINTER(TopoDesc), C.POINTER(C.c_uint16),
                                                   C.POINTER(C.c_float), C.POINTER(C.c_float),
                                                   C.POINTER(C.c_float), C.POINTER(C.c_float)]),
        "msbg_gpu_pressure_level_size": (i32, [vp, i32, C.POINTER(C.c_int64)]),
        "msbg_gpu_pressure_diagonal": (i32, [vp, i32, C.POINTER(C.c_float), C.c_int64]),
        "msbg_gpu_matvec": (i32, [vp, i32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int64]),
        "msbg_gpu_residual": (i32, [vp, i32, C.POINTER(C.c_float), C.POINTER(C.c_float),
                                    C.POINTER(C.c_float), C.c_int64]),
        "msbg_gpu_restrict": (i32, [vp, i32, C.POINTER(C.c_float), C.c_int64, C.POINTER(C.c_float),
                                    C.c_int64]),
        "msbg_gpu_prolongate": (i32, [vp, i32, C.POINTER(C.c_float), C.c_int64,
                                      C.POINTER(C.c_float), C.c_int64, C.c_float]),
        "msbg_gpu_relax": (i32, [vp, i32, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int64,
                                 i32, i32, i32, i32, C.c_float]),
        "msbg_gpu_vcycle": (i32, [vp, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_int64, i32,
                                  i32, i32, C.c_float]),
        "msbg_gpu_pressure_host_check": (i32, [C.POINTER(TopoDesc), C.POINTER(PressureCallbacks),
                                               C.POINTER(C.c_float), C.POINTER(C.c_double),
                                               C.POINTER(C.c_int), C.POINTER(C.c_int64),
                                               C.POINTER(C.c_double)]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


class PressureScene:
    """Seeded free-surface pressure problem (include/msbg_scene.h)."""

    def __init__(self, res, bsx0, n_levels, z_liquid=0.4, n_spheres=32, r_min=0.03, r_max=0.1,
                 n_cuboids=8, n_modes=16, k_max=8, band=64.0, seed=2024, wave_amp=0.0,
                 n_waves=0):
        L = scene_lib()
        self._L = L
        self.res, self.bsx0, self.n_levels = res, bsx0, n_levels
        self.h = L.msbg_scene_pressure_create_wavy(res, bsx0, n_levels, z_liquid, wave_amp,
                                                   n_waves, n_spheres, r_min, r_max, n_cuboids,
                                                   n_modes, k_max, band, seed)
        if not self.h:
            raise MsbgError(5, "scene")
        nb = (res // bsx0) ** 3
        self.block_levels = np.zeros(nb, np.int32)
        L.msbg_scene_pressure_block_levels(self.h, _p(self.block_levels, C.c_int))

    def callbacks(self):
        L = self._L
        return PressureCallbacks(C.cast(L.msbg_scene_cell_type, C.c_void_p).value,
                                 C.cast(L.msbg_scene_face_coeff, C.c_void_p).value,
                                 C.cast(L.msbg_scene_rhs, C.c_void_p).value, self.h)

    def packed_size(self):
        return int(sum((self.bsx0 >> int(l)) ** 3 for l in self.block_levels))

    def arrays(self, pinned=False):
        """The scene as the per-cell arrays of Context.pressure_prepare_arrays:
        (flags uint16, [faceX, faceY, faceZ] float32, rhs float32); pinned:
        in page-locked host memory (the prepare then copies them to the GPU
        by DMA straight from there)."""
        n = self.packed_size()
        alloc = pinned_empty if pinned else np.empty
        flags = alloc(n, np.uint16)
        face = [alloc(n, np.float32) for _ in range(3)]
        rhs = alloc(n, np.float32)
        rc = self._L.msbg_scene_pressure_arrays(self.h, _p(flags, C.c_uint16),
                                                *[_p(f, C.c_float) for f in face],
                                                _p(rhs, C.c_float))
        if rc:
            raise MsbgError(rc, "scene arrays")
        return flags, face, rhs

    def close(self):
        if self.h:
            self._L.msbg_scene_pressure_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_params(**kw):
    L = lib()
    _pressure_sigs(L)
    p = SolveParams()
    L.msbg_gpu_solve_params_default(C.byref(p))
    for k, v in kw.items():
        setattr(p, k, v)
    return p


def _ctx_pressure_prepare(self, scene, domain_bc=None):
    """msbg_gpu_pressure_prepare with the scene's callbacks; domain_bc: six
    DBC_OPEN / DBC_SOLID values (-x, +x, -y, +y, -z, +z), or None for the
    reference's operator (lower domain faces open with the callback's
    coefficient, upper faces closed)."""
    _pressure_sigs(self._L)
    self._bl_p = np.ascontiguousarray(scene.block_levels, np.int32)
    self._dbc_p = None if domain_bc is None else np.ascontiguousarray(domain_bc, np.int32)
    d = TopoDesc(scene.res, scene.res, scene.res, scene.bsx0, scene.n_levels,
                 _p(self._bl_p, C.c_int), _p(self._dbc_p, C.c_int))
    cb = scene.callbacks()
    self._check(self._L.msbg_gpu_pressure_prepare(self._h, C.byref(d), C.byref(cb)),
                "pressure_prepare")


def _ctx_pressure_solve(self, params=None, **kw):
    p = params or solve_params(**kw)
    info = SolveInfo()
    self._check(self._L.msbg_gpu_pressure_solve(self._h, C.byref(p), C.byref(info)),
                "pressure_solve")
    self._last_launches = info.kernelLaunches
    return info


def _ctx_pressure_profile(self, what, reps, inner=2):
    ms = C.c_double()
    by = C.c_double()
    self._check(self._L.msbg_gpu_pressure_profile(self._h, what, reps, inner, C.byref(ms),
                                                  C.byref(by)), "pressure_profile")
    return ms.value, by.value


def count_liquid_cells(scene):
    """Liquid cells of MG level 0 of a scene (host-side hierarchy build, no GPU)."""
    L = lib()
    _pressure_sigs(L)
    bl = np.ascontiguousarray(scene.block_levels, np.int32)
    d = TopoDesc(scene.res, scene.res, scene.res, scene.bsx0, scene.n_levels,
                 _p(bl, C.c_int))
    cb = scene.callbacks()
    nm = C.c_int()
    fluid = np.zeros(32, np.int64)
    rc = L.msbg_gpu_pressure_host_check(C.byref(d), C.byref(cb), None, None, C.byref(nm),
                                        _p(fluid, C.c_int64), None)
    if rc:
        raise MsbgError(rc, "host check")
    return int(fluid[0])


def _ctx_pressure_download(self, rhs=False, fp64=False, out=None):
    """The pressure (or the rhs) in the block layout; out: a float32 array of
    the packed size to fill instead of a new one."""
    n = C.c_int64()
    self._check(self._L.msbg_gpu_pressure_packed_size(self._h, C.byref(n)), "packed_size")
    if fp64:
        out = np.zeros(n.value, np.float64)
        self._check(self._L.msbg_gpu_pressure_download64(self._h, _p(out, C.c_double), n.value),
                    "pressure_download64")
        return out
    if out is None:
        out = np.zeros(n.value, np.float32)
    elif out.dtype != np.float32 or out.size != n.value or not out.flags.c_contiguous:
        raise ValueError("out: contiguous float32 array of the packed size")
    fn = self._L.msbg_gpu_pressure_download_rhs if rhs else self._L.msbg_gpu_pressure_download
    self._check(fn(self._h, _p(out, C.c_float), n.value), "pressure_download")
    return out


def _f32(a):
    return np.ascontiguousarray(a, np.float32)


def _ctx_pressure_prepare_arrays(self, res, bsx0, n_levels, block_levels, flags, face, rhs=None,
                                 domain_bc=None):
    """msbg_gpu_pressure_prepare_arrays: per-cell flags, lower-face coefficients
    face[3] and rhs in the packed block layout of MG level 0; domain_bc as in
    pressure_prepare."""
    _pressure_sigs(self._L)
    self._bl_p = np.ascontiguousarray(block_levels, np.int32)
    self._dbc_p = None if domain_bc is None else np.ascontiguousarray(domain_bc, np.int32)
    d = TopoDesc(res, res, res, bsx0, n_levels, _p(self._bl_p, C.c_int), _p(self._dbc_p, C.c_int))
    fl = np.ascontiguousarray(flags, np.uint16)
    fx, fy, fz = (_f32(f) for f in face)
    rh = None if rhs is None else _f32(rhs)
    self._check(self._L.msbg_gpu_pressure_prepare_arrays(
        self._h, C.byref(d), _p(fl, C.c_uint16), _p(fx, C.c_float), _p(fy, C.c_float),
        _p(fz, C.c_float), _p(rh, C.c_float)), "pressure_prepare_arrays")


def _ctx_level_size(self, level_mg):
    n = C.c_int64()
    self._check(self._L.msbg_gpu_pressure_level_size(self._h, level_mg, C.byref(n)), "level_size")
    return n.value


def _ctx_diagonal(self, level_mg=0):
    out = np.zeros(self.level_size(level_mg), np.float32)
    self._check(self._L.msbg_gpu_pressure_diagonal(self._h, level_mg, _p(out, C.c_float),
                                                   len(out)), "pressure_diagonal")
    return out


def _ctx_matvec(self, level_mg, x):
    x = _f32(x)
    y = np.zeros_like(x)
    self._check(self._L.msbg_gpu_matvec(self._h, level_mg, _p(x, C.c_float), _p(y, C.c_float),
                                        len(x)), "matvec")
    return y


def _ctx_residual(self, level_mg, x, b):
    x, b = _f32(x), _f32(b)
    r = np.zeros_like(x)
    self._check(self._L.msbg_gpu_residual(self._h, level_mg, _p(x, C.c_float), _p(b, C.c_float),
                                          _p(r, C.c_float), len(x)), "residual")
    return r


def _ctx_restrict(self, level_mg_coarse, fine):
    fine = _f32(fine)
    coarse = np.zeros(self.level_size(level_mg_coarse), np.float32)
    self._check(self._L.msbg_gpu_restrict(self._h, level_mg_coarse, _p(fine, C.c_float), len(fine),
                                          _p(coarse, C.c_float), len(coarse)), "restrict")
    return coarse


def _ctx_prolongate(self, level_mg_fine, coarse, fine, scale=1.0):
    coarse = _f32(coarse)
    out = _f32(fine).copy()
    self._check(self._L.msbg_gpu_prolongate(self._h, level_mg_fine, _p(coarse, C.c_float),
                                            len(coarse), _p(out, C.c_float), len(out), scale),
                "prolongate")
    return out


def _ctx_relax(self, level_mg, x, b, n_iter, reverse=0, inner=3, mode=0, omega=1.0):
    out = _f32(x).copy()
    b = _f32(b)
    self._check(self._L.msbg_gpu_relax(self._h, level_mg, _p(out, C.c_float), _p(b, C.c_float),
                                       len(out), n_iter, reverse, inner, mode, omega), "relax")
    return out


def _ctx_vcycle(self, r, n_pre=2, n_post=2, inner=3, coarse_scale=1.8):
    r = _f32(r)
    z = np.zeros_like(r)
    self._check(self._L.msbg_gpu_vcycle(self._h, _p(r, C.c_float), _p(z, C.c_float), len(r), n_pre,
                                        n_post, inner, coarse_scale), "vcycle")
    return z


Context.pressure_prepare_arrays = _ctx_pressure_prepare_arrays
Context.level_size = _ctx_level_size
Context.diagonal = _ctx_diagonal
Context.matvec = _ctx_matvec
Context.residual = _ctx_residual
Context.restrict = _ctx_restrict
Context.prolongate = _ctx_prolongate
Context.relax = _ctx_relax
Context.vcycle = _ctx_vcycle
Context.pressure_prepare = _ctx_pressure_prepare
Context.pressure_solve = _ctx_pressure_solve
Context.pressure_download = _ctx_pressure_download
Context.pressure_profile = _ctx_pressure_profile
Context.last_solve_launches = lambda self: getattr(self, "_last_launches", None)


from .learned import Cnn, collect_correction_pairs, collect_training_pairs, train_cnn  # noqa: E402,F401


# ---------------------------------------------------------------------------
# FLIP transfers around the pressure solve (single-level grids)
# ---------------------------------------------------------------------------
FLIP_VEL, FLIP_VEL_OLD, FLIP_BETA, FLIP_MASS = 0, 1, 2, 3
# msbg_flip_particle = FlipParticle (src/flip_sim.h:48): 28 bytes
FLIP_PARTICLE = np.dtype([("pos", "<f4", (3,)), ("vel", "<f4", (3,)), ("phase", "<i4")])
assert FLIP_PARTICLE.itemsize == 28


class FlipParams(C.Structure):
    _fields_ = [("rhoL", C.c_float), ("rhoG", C.c_float), ("massEps", C.c_float),
                ("betaMin", C.c_float), ("alphaPhi", C.c_float), ("particlesPerVoxel", C.c_int)]


def flip_params(rhoL=1000.0, rhoG=1.0, massEps=1e-5, betaMin=1e-6, alphaPhi=1.0,
                particlesPerVoxel=8):
    """FlipConfig's defaults (src/flip_sim.h:29-45)."""
    return FlipParams(rhoL, rhoG, massEps, betaMin, alphaPhi, particlesPerVoxel)


def _flip_sigs(L):
    if getattr(L, "_flip_sig", False):
        return
    vp, i32, f32 = C.c_void_p, C.c_int, C.c_float
    sig = {
        "msbg_gpu_flip_p2g": (i32, [vp, vp, C.c_int64, C.POINTER(FlipParams),
                                    C.POINTER(C.c_int), C.POINTER(C.c_int64)]),
        "msbg_gpu_flip_gravity": (i32, [vp, f32, f32, f32]),
        "msbg_gpu_flip_pressure_gradient": (i32, [vp, C.POINTER(C.c_float), f32, f32]),
        "msbg_gpu_flip_g2p": (i32, [vp, vp, C.c_int64, f32]),
        "msbg_gpu_flip_channel": (i32, [vp, i32, C.POINTER(C.c_float), C.c_int64, i32]),
        "msbg_gpu_flip_p2g_device": (i32, [vp, vp, C.c_int64, C.POINTER(FlipParams),
                                           C.POINTER(C.c_int), C.POINTER(C.c_int64)]),
        "msbg_gpu_flip_g2p_device": (i32, [vp, vp, C.c_int64, f32]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    L._flip_sig = True


def _ctx_flip_p2g(self, particles, params=None):
    """msbg_gpu_flip_p2g after set_topology; returns the active block ids."""
    _flip_sigs(self._L)
    p = np.ascontiguousarray(particles, FLIP_PARTICLE)
    prm = params or flip_params()
    act = np.zeros(max(getattr(self, "n_blocks", 0), 1), np.int32)
    nb = C.c_int64()
    self._check(self._L.msbg_gpu_flip_p2g(self._h, p.ctypes.data, len(p), C.byref(prm),
                                          _p(act, C.c_int), C.byref(nb)), "flip_p2g")
    return act[:nb.value]


def _ctx_flip_gravity(self, gravity, dt, mass_eps=1e-5):
    _flip_sigs(self._L)
    self._check(self._L.msbg_gpu_flip_gravity(self._h, gravity, dt, mass_eps), "flip_gravity")


def _ctx_flip_pressure_gradient(self, pressure, dt, mass_eps=1e-5):
    _flip_sigs(self._L)
    p = _f32(pressure)
    self._check(self._L.msbg_gpu_flip_pressure_gradient(self._h, _p(p, C.c_float), dt,
                                                        mass_eps), "flip_pressure_gradient")


def _ctx_flip_g2p(self, particles, alpha=0.95):
    """msbg_gpu_flip_g2p on a FLIP_PARTICLE array, in place."""
    _flip_sigs(self._L)
    if not (particles.flags.c_contiguous and particles.dtype == FLIP_PARTICLE):
        raise ValueError("particles: contiguous FLIP_PARTICLE array")
    self._check(self._L.msbg_gpu_flip_g2p(self._h, particles.ctypes.data, len(particles), alpha),
                "flip_g2p")


def _ctx_flip_channel(self, which, n_voxels, data=None):
    """Get (data None) or set a FLIP channel: 3 floats per voxel, 1 for the mass."""
    _flip_sigs(self._L)
    comps = 1 if which == FLIP_MASS else 3
    if data is None:
        out = np.empty(comps * n_voxels, np.float32)
        self._check(self._L.msbg_gpu_flip_channel(self._h, which, _p(out, C.c_float), len(out),
                                                  1), "flip_channel")
        return out
    d = _f32(data).reshape(-1)
    self._check(self._L.msbg_gpu_flip_channel(self._h, which, _p(d, C.c_float), len(d), 0),
                "flip_channel")


def _ctx_flip_p2g_device(self, dev_ptr, n_particles, params=None):
    """msbg_gpu_flip_p2g_device on particles at device address dev_ptr."""
    _flip_sigs(self._L)
    prm = params or flip_params()
    nb = C.c_int64()
    self._check(self._L.msbg_gpu_flip_p2g_device(self._h, dev_ptr, n_particles, C.byref(prm),
                                                 None, C.byref(nb)), "flip_p2g_device")
    return nb.value


def _ctx_flip_g2p_device(self, dev_ptr, n_particles, alpha=0.95):
    _flip_sigs(self._L)
    self._check(self._L.msbg_gpu_flip_g2p_device(self._h, dev_ptr, n_particles, alpha),
                "flip_g2p_device")


def _mr_sigs(L):
    if getattr(L, "_mr_sig", False):
        return
    vp, i32, f32 = C.c_void_p, C.c_int, C.c_float
    sig = {
        "msbg_gpu_flip_mr_dist": (i32, [vp, vp, C.c_int64, vp, C.c_int64]),
        "msbg_gpu_flip_mr_channel": (i32, [vp, i32, C.POINTER(C.c_float), C.c_int64, i32]),
        "msbg_gpu_flip_g2p_mr": (i32, [vp, vp, C.c_int64, f32]),
        "msbg_gpu_flip_g2p_mr_device": (i32, [vp, vp, C.c_int64, f32]),
        "msbg_gpu_flip_downsample_velocity": (i32, [vp, i32, vp, vp, C.c_int64, vp, C.c_int64]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args
    L._mr_sig = True


def packed_voxels(bsx0, block_level):
    """Voxels of the packed layout: (bsx0 >> level)^3 per block."""
    bl = np.asarray(block_level, np.int64)
    return int(((bsx0 >> bl) ** 3).sum())


def _ctx_flip_mr_dist(self, n_levels):
    """msbg_gpu_flip_mr_dist: (packed uint16 distances, kinds [n_levels, nBlocks])."""
    _mr_sigs(self._L)
    n = packed_voxels(self._bsx0, self._levels)
    dist = np.zeros(n, np.uint16)
    kind = np.zeros((n_levels, len(self._levels)), np.int8)
    self._check(self._L.msbg_gpu_flip_mr_dist(self._h, dist.ctypes.data, n, kind.ctypes.data,
                                              kind.size), "flip_mr_dist")
    return dist, kind


def _ctx_flip_mr_channel(self, which, data=None):
    """Get (data None) or set a mixed-resolution velocity channel (3 floats per
    packed voxel)."""
    _mr_sigs(self._L)
    n = 3 * packed_voxels(self._bsx0, self._levels)
    if data is None:
        out = np.empty(n, np.float32)
        self._check(self._L.msbg_gpu_flip_mr_channel(self._h, which, _p(out, C.c_float), n, 1),
                    "flip_mr_channel")
        return out
    d = _f32(data).reshape(-1)
    self._check(self._L.msbg_gpu_flip_mr_channel(self._h, which, _p(d, C.c_float), len(d), 0),
                "flip_mr_channel")


def _ctx_flip_g2p_mr(self, particles, alpha=0.95):
    """msbg_gpu_flip_g2p_mr on a FLIP_PARTICLE array, in place."""
    _mr_sigs(self._L)
    if not (particles.flags.c_contiguous and particles.dtype == FLIP_PARTICLE):
        raise ValueError("particles: contiguous FLIP_PARTICLE array")
    self._check(self._L.msbg_gpu_flip_g2p_mr(self._h, particles.ctypes.data, len(particles),
                                             alpha), "flip_g2p_mr")


def _ctx_flip_g2p_mr_device(self, dev_ptr, n_particles, alpha=0.95):
    _mr_sigs(self._L)
    self._check(self._L.msbg_gpu_flip_g2p_mr_device(self._h, dev_ptr, n_particles, alpha),
                "flip_g2p_mr_device")


def _ctx_flip_downsample_velocity(self, level_mg, flags, src):
    """msbg_gpu_flip_downsample_velocity: MG level level_mg - 1 (src) to
    level_mg, with that level's cell flags; returns dst."""
    _mr_sigs(self._L)
    lv = np.maximum(np.asarray(self._levels, np.int64), level_mg)
    n = int(((self._bsx0 >> lv) ** 3).sum())
    fl = np.ascontiguousarray(flags, np.uint16)
    s = _f32(src).reshape(-1)
    dst = np.empty(3 * n, np.float32)
    self._check(self._L.msbg_gpu_flip_downsample_velocity(self._h, level_mg, fl.ctypes.data,
                                                          s.ctypes.data, len(s), dst.ctypes.data,
                                                          len(dst)), "flip_downsample_velocity")
    return dst


Context.flip_downsample_velocity = _ctx_flip_downsample_velocity
Context.flip_mr_dist = _ctx_flip_mr_dist
Context.flip_mr_channel = _ctx_flip_mr_channel
Context.flip_g2p_mr = _ctx_flip_g2p_mr
Context.flip_g2p_mr_device = _ctx_flip_g2p_mr_device
Context.flip_p2g_device = _ctx_flip_p2g_device
Context.flip_g2p_device = _ctx_flip_g2p_device
Context.flip_p2g = _ctx_flip_p2g
Context.flip_gravity = _ctx_flip_gravity
Context.flip_pressure_gradient = _ctx_flip_pressure_gradient
Context.flip_g2p = _ctx_flip_g2p
Context.flip_channel = _ctx_flip_channel


def flip_particles(res, bsx, z_liquid=0.4, ppv=8, air_ppv=1, air_band=8, seed=7, vel_scale=1.0):
    """Seeded FLIP particles on a res^3 grid: ppv liquid particles jittered in
    every cell below z_liquid * res, air_ppv air particles in the air_band
    cells above it; velocities from three seeded sinusoids.  Returns a
    FLIP_PARTICLE array."""
    rng = np.random.default_rng(seed)
    zl = int(z_liquid * res)
    out = []
    for zlo, zhi, n, phase in ((0, zl, ppv, 0), (zl, min(res, zl + air_band), air_ppv, 1)):
        if zhi <= zlo or n <= 0:
            continue
        cz, cy, cx = np.meshgrid(np.arange(zlo, zhi), np.arange(res), np.arange(res),
                                 indexing="ij")
        cells = np.stack([cx.ravel(), cy.ravel(), cz.ravel()], 1).astype(np.float32)
        pos = np.repeat(cells, n, 0) + rng.random((len(cells) * n, 3), dtype=np.float32)
        a = rng.standard_normal((3, 3)).astype(np.float32)
        vel = np.stack([np.sin(2 * np.pi * (pos @ a[i]) / res) for i in range(3)], 1) * vel_scale
        p = np.empty(len(pos), FLIP_PARTICLE)
        p["pos"] = pos
        p["vel"] = vel.astype(np.float32)
        p["phase"] = phase
        out.append(p)
    return np.concatenate(out)


# ---------------------------------------------------------------------------
# Particle splatting into a 16-bit render-density channel
# ---------------------------------------------------------------------------
SPLAT_RAW = 1


class SplatParams(C.Structure):
    _fields_ = [("rParticle", C.c_float), ("nbDist", C.c_float), ("flags", C.c_int)]


def _splat_sigs(L):
    if getattr(L, "_splat_sig", False):
        return
    vp, i32 = C.c_void_p, C.c_int
    for name in ("msbg_gpu_splat_particles", "msbg_gpu_splat_particles_device"):
        fn = getattr(L, name)
        fn.restype = i32
        fn.argtypes = [vp, i32, vp, C.c_int64, C.POINTER(SplatParams), vp, vp]
    L._splat_sig = True


def _ctx_splat(self, chan, pos, r_particle=2.0, nb_dist=2.0, kind=None, raw=False):
    """msbg_gpu_splat_particles after set_topology: creates 16-bit channel
    `chan` from particle positions [n, 3]; returns the block kinds used."""
    _splat_sigs(self._L)
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    prm = SplatParams(r_particle, nb_dist, SPLAT_RAW if raw else 0)
    kout = np.zeros(max(getattr(self, "n_blocks", 0), 1), np.int8)
    k = None if kind is None else np.ascontiguousarray(kind, np.int8)
    self._check(self._L.msbg_gpu_splat_particles(self._h, chan, p.ctypes.data, len(p),
                                                 C.byref(prm),
                                                 None if k is None else k.ctypes.data,
                                                 kout.ctypes.data), "splat_particles")
    return kout


def _ctx_splat_device(self, chan, dev_ptr, n_particles, r_particle=2.0, nb_dist=2.0, kind=None,
                      raw=False):
    """msbg_gpu_splat_particles_device on positions at device address dev_ptr."""
    _splat_sigs(self._L)
    prm = SplatParams(r_particle, nb_dist, SPLAT_RAW if raw else 0)
    kout = np.zeros(max(getattr(self, "n_blocks", 0), 1), np.int8)
    k = None if kind is None else np.ascontiguousarray(kind, np.int8)
    self._check(self._L.msbg_gpu_splat_particles_device(self._h, chan, dev_ptr, n_particles,
                                                        C.byref(prm),
                                                        None if k is None else k.ctypes.data,
                                                        kout.ctypes.data), "splat_particles")
    return kout


Context.splat = _ctx_splat
Context.splat_device = _ctx_splat_device


def splat_base_cloud(n_base, seed=11):
    """A seeded stand-in for the demo's PLY model: n_base points near an
    ellipsoid surface, float32 [n_base, 3]."""
    rng = np.random.default_rng(seed)
    v = rng.normal(size=(n_base, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return (v * np.array([1.0, 0.7, 0.5]) + 0.05 * rng.normal(size=(n_base, 3))).astype(np.float32)


def splat_demo_particles(res3, n_base, seed=11, test_case=1, base=None):
    """Seeded particles built the way the reference's demo builds its
    bunny-of-bunnies (src/msbg_demo.cpp:339-385): n_base instances of a base
    cloud of n_base points (splat_base_cloud, or `base`), instance i at
    0.2 * sMax + 0.6 * sMax * b_i and scaled by 0.01 * sMin (0.005 for test
    case 2), b the base cloud normalised by its bounding box.  Returns
    float32 [n_base^2, 3]."""
    v = splat_base_cloud(n_base, seed) if base is None else np.asarray(base, np.float32)
    bmin = v.min(0)
    span = (v.max(0) - bmin).max()
    b = ((v - bmin) * np.float32(1.0 / span)).astype(np.float32)
    smax, smin = max(res3), min(res3)
    scale = np.float32(smin * (0.005 if test_case == 2 else 0.01))
    centres = (np.float32(smax * 0.2) + np.float32(0.6) * (np.float32(smax) * b)).astype(np.float32)
    pos = centres[:, None, :] + scale * b[None, :, :]
    return pos.reshape(-1, 3).astype(np.float32)


def pinned_empty(shape, dtype):
    """An uninitialised numpy array in page-locked host memory (a pinned torch
    tensor's storage; the array keeps the tensor alive)."""
    import torch
    dt = np.dtype(dtype)
    t = torch.empty(int(np.prod(shape)) * dt.itemsize, dtype=torch.uint8, pin_memory=True)
    a = t.numpy().view(dt).reshape(shape)
    return a
