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
# reference channel ids (src/msbg.h enum order is not needed: the harness takes ids)
CH = {}


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
        L.ref_ps_block_info.argtypes = [vp, C.c_int, C.POINTER(C.c_int), C.POINTER(C.c_int)]
        L.ref_ps_packed_size.restype = C.c_longlong
        L.ref_ps_packed_size.argtypes = [vp, C.c_int]
        L.ref_ps_channel.argtypes = [vp, C.c_int, C.c_int, C.POINTER(C.c_float), C.c_int, C.c_int]
        L.ref_ps_multiply.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.ref_ps_relax.argtypes = [vp, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]
        L.ref_ps_downsample.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.ref_ps_prolongate.argtypes = [vp, C.c_int, C.c_int, C.c_int]
        L.ref_ps_vcycle.argtypes = [vp] + [C.c_int] * 7
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

    def solve(self, n_pre=2, n_post=2, n_coarse=24, max_iter=500, tol=1e-6):
        rr = C.c_float()
        secs = C.c_double()
        it = self._L.ref_ps_solve(self.h, n_pre, n_post, n_coarse, max_iter, tol, C.byref(rr),
                                  C.byref(secs))
        return it, rr.value, secs.value
