"""ctypes driver of the reference FLIP pressure solver (TEST INFRASTRUCTURE ONLY).

Runs the compiled reference (oracle/_ref/libmsbg_ref.so): preparePressureSolveFLIP
with the caller's scene callbacks, then its solver pieces (src/msbg3.cpp).
Used for per-kernel parity tests and as the timed CPU baseline.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

import oracle

DBC_OPEN, DBC_SOLID = 0, 1
# reference channel ids (src/msbg.h:279-328) and the harness's pseudo channels
CH_FLOAT_1, CH_DIVERGENCE, CH_PRESSURE, CH_FLOAT_2, CH_FLOAT_3, CH_DIAGONAL, CH_FLOAT_6 = (
    1, 2, 3, 6, 7, 13, 36)
CH_FACE = (-1, -2, -3)  # CH_FACE_AREA dir 0, 1, 2
CH_FLAGS = -10          # CH_CELL_FLAGS
CH_VEC3_2, CH_VEC3_4 = 21, 23  # vector channels (src/msbg.h:302-305)
CELL_SOLID, CELL_FIXED, CELL_VOID = 0x1, 0x2, 0x1000


def _lib():
    L = oracle.ref()
    if not hasattr(L, "_ps"):
        vp = C.c_void_p
        L.ref_ps_create.restype = vp
        L.ref_ps_create.argtypes = [C.c_int] * 5 + [C.POINTER(C.c_int), C.POINTER(C.c_int), vp, vp,
                                                    vp, vp, C.POINTER(C.c_double)]
        L.ref_ps_destroy.argtypes = [vp]
        L.ref_ps_omega.restype = C.c_float
        L.ref_ps_omega.argtypes = [vp]
        L.ref_ps_num_levels.restype = C.c_int
        L.ref_ps_num_levels.argtypes = [vp]
        L.ref_ps_block_info.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.ref_ps_packed_size.restype = C.c_longlong
        L.ref_ps_packed_size.argtypes = [vp, C.c_int]
        L.ref_ps_channel.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_float), C.c_int, C.c_int]
        L.ref_ps_multiply.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.ref_ps_relax.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.ref_ps_downsample.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.ref_ps_prolongate.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.ref_ps_vcycle.argtypes = [vp] + [C.c_int] * 7
        L.ref_ps_vec_channel.restype = C.c_int
        L.ref_ps_vec_channel.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_float), C.c_int,
                                         C.c_int]
        L.ref_ps_downsample_velocity.restype = C.c_int
        L.ref_ps_downsample_velocity.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.ref_ps_solve.restype = C.c_int
        L.ref_ps_solve.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_float,
                                   C.POINTER(C.c_float), C.POINTER(C.c_double)]
        L._ps = True
    return L


class RefPressure:
    """A prepared reference pressure problem (MultiresSparseGrid + FLIP setup)."""

    def __init__(self, scene, dom_bc=(DBC_SOLID,) * 6):
        L = _lib()
        self._L = L
        self.scene = scene
        cb = scene.callbacks()
        bl = np.ascontiguousarray(scene.block_levels, np.int32)
        bc = np.ascontiguousarray(dom_bc, np.int32)
        secs = C.c_double()
        self.h = L.ref_ps_create(scene.res, scene.res, scene.res, scene.bsx0, scene.n_levels,
                                 bl.ctypes.data_as(C.POINTER(C.c_int)),
                                 bc.ctypes.data_as(C.POINTER(C.c_int)), cb.sampleCellType,
                                 cb.sampleFaceCoeff, cb.sampleRhs, cb.user, C.byref(secs))
        if not self.h:
            raise RuntimeError("ref_ps_create failed")
        self.prep_seconds = secs.value

    def close(self):
        if self.h:
            self._L.ref_ps_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def omega(self):
        return self._L.ref_ps_omega(self.h)

    def num_levels(self):
        return self._L.ref_ps_num_levels(self.h)

    def block_levels(self, level_mg):
        nb = len(self.scene.block_levels)
        lev = np.zeros(nb, np.int32)
        flg = np.zeros(nb, np.int32)
        self._L.ref_ps_block_info(self.h, level_mg, lev.ctypes.data_as(C.POINTER(C.c_int)),
                                  flg.ctypes.data_as(C.POINTER(C.c_int)))
        return lev, flg

    def packed_size(self, level_mg):
        return int(self._L.ref_ps_packed_size(self.h, level_mg))

    def get(self, ch, level_mg=0):
        """Channel ch of MG level level_mg in the packed block layout (missing
        blocks read 0; flags of missing blocks read -1)."""
        out = np.zeros(self.packed_size(level_mg), np.float32)
        self._L.ref_ps_channel(self.h, ch, level_mg, out.ctypes.data_as(C.POINTER(C.c_float)), 1, 0)
        return out

    def set(self, ch, data, level_mg=0):
        d = np.ascontiguousarray(data, np.float32)
        assert len(d) == self.packed_size(level_mg)
        self._L.ref_ps_channel(self.h, ch, level_mg, d.ctypes.data_as(C.POINTER(C.c_float)), 0, 1)

    def multiply(self, level_mg, ch_x, ch_dst, ch_b=None):
        """multiplyLaplacianMatrixOpt: ch_dst = A x, or b - A x with ch_b."""
        self._L.ref_ps_multiply(self.h, level_mg, ch_x, ch_b if ch_b is not None else -1, ch_dst,
                                1 if ch_b is not None else 0)

    def relax(self, level_mg, ch_x, ch_b, ch_tmp, n_iter, reverse=0):
        self._L.ref_ps_relax(self.h, level_mg, ch_x, ch_b, ch_tmp, n_iter, reverse)

    def downsample(self, level_mg_coarse, ch_src, ch_dst):
        self._L.ref_ps_downsample(self.h, level_mg_coarse, ch_src, ch_dst)

    def prolongate(self, level_mg_fine, ch_src, ch_dst):
        self._L.ref_ps_prolongate(self.h, level_mg_fine, ch_src, ch_dst)

    def get_vec(self, ch, level_mg=0):
        """Vector channel ch (CH_VEC3_*) of MG level level_mg, packed, 3 floats
        per voxel."""
        out = np.zeros(3 * self.packed_size(level_mg), np.float32)
        rc = self._L.ref_ps_vec_channel(self.h, ch, level_mg,
                                        out.ctypes.data_as(C.POINTER(C.c_float)), 1, 0)
        if rc:
            raise RuntimeError(f"ref_ps_vec_channel rc={rc}")
        return out

    def set_vec(self, ch, data, level_mg=0):
        d = np.ascontiguousarray(data, np.float32)
        assert len(d) == 3 * self.packed_size(level_mg)
        rc = self._L.ref_ps_vec_channel(self.h, ch, level_mg,
                                        d.ctypes.data_as(C.POINTER(C.c_float)), 0, 1)
        if rc:
            raise RuntimeError(f"ref_ps_vec_channel rc={rc}")

    def downsample_velocity(self, level_mg, ch_src, ch_dst):
        """downsampleVelocity (src/msbg4.cpp:2035): MG level level_mg - 1 to level_mg."""
        rc = self._L.ref_ps_downsample_velocity(self.h, level_mg, ch_src, ch_dst)
        if rc:
            raise RuntimeError(f"ref_ps_downsample_velocity rc={rc}")

    def level0_arrays(self):
        """The reference's prepared level-0 inputs (preparePressureSolveFLIPLevel0_,
        src/msbg3.cpp:2472-2584): cell flags, lower-face coefficients per
        direction and the rhs, in the packed block layout."""
        flags = self.get(CH_FLAGS).astype(np.int64)
        assert (flags >= 0).all(), "every level-0 block holds flags after the prepare"
        return (flags.astype(np.uint16), [self.get(c) for c in CH_FACE], self.get(CH_DIVERGENCE))

    def liquid(self, level_mg=0):
        """Cells the reference solves for: not SOLID, VOID or FIXED."""
        fl = self.get(CH_FLAGS, level_mg).astype(np.int64)
        return (fl >= 0) & ((fl & (CELL_SOLID | CELL_VOID | CELL_FIXED)) == 0)

    def array_scene(self):
        """oracle.ArrayScene over the reference's own prepared level-0 inputs."""
        flags, face, rhs = self.level0_arrays()
        s = self.scene
        return oracle.ArrayScene(s.res, s.bsx0, s.n_levels, s.block_levels, flags, face, rhs)

    def solve(self, n_pre=2, n_post=2, n_coarse=24, max_iter=500, tol=1e-6):
        rr = C.c_float()
        secs = C.c_double()
        it = self._L.ref_ps_solve(self.h, n_pre, n_post, n_coarse, max_iter, tol, C.byref(rr),
                                  C.byref(secs))
        return it, rr.value, secs.value
