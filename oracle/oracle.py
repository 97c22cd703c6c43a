"""ctypes loader of the oracle libraries (TEST INFRASTRUCTURE ONLY).

- ``libmsbg_oracle.so``: the C restatement (oracle/msbg_oracle.c).
- ``libmsbg_ref.so``: the reference MSBG core compiled from its own sources
  plus oracle/ref/ref_harness.cpp (present only where it was built).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg use this
module; the GPU product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(OUT, "libmsbg_oracle.so")
REF_SO = os.path.join(OUT, "libmsbg_ref.so")

# The reference tree the recipe compiles: $MSBG_REFERENCE, else its usual
# mount point.  Only the build reads it; the prebuilt libraries need no tree.
REFERENCE_ROOT = os.environ.get("MSBG_REFERENCE", "/root/reference")

_oracle = None
_ref = None


def _p(a, ct):
    return a.ctypes.data_as(C.POINTER(ct)) if a is not None else None


def build_oracle():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def build_ref(ref_root=REFERENCE_ROOT):
    if not os.path.isdir(os.path.join(ref_root, "src")):
        return False
    subprocess.run(["make", "-s", "-j8", "-C", HERE, "ref", f"REF_ROOT={ref_root}"], check=True)
    # the reference's particle-splatting demo with its capture hooks
    subprocess.run(["make", "-s", "-C", HERE, "splat", f"REF_ROOT={ref_root}"], check=True)
    # the INTEGRATION.md snippets compiled against the reference headers
    # (needs msbg-flip_b200/libmsbg_gpu.so, built before the oracle)
    subprocess.run(["make", "-s", "-C", HERE, "integ", f"REF_ROOT={ref_root}"], check=True)
    return True


def oracle():
    global _oracle
    if _oracle is None:
        if not os.path.exists(ORACLE_SO):
            build_oracle()
        L = C.CDLL(ORACLE_SO)
        L.oracle_mcf.restype = C.c_int
        L.oracle_mcf.argtypes = [C.c_int] * 4 + [C.POINTER(C.c_int8), C.c_float, C.c_float,
                                                 C.POINTER(C.c_float), C.POINTER(C.c_int),
                                                 C.c_int, C.c_int, C.c_float, C.c_int, C.c_int]
        _oracle = L
    return _oracle


def ref_available():
    return os.path.exists(REF_SO)


INTEG_SO = os.path.join(OUT, "libmsbg_integ.so")
_integ = None


def integ_available():
    return os.path.exists(INTEG_SO)


def integ():
    """The INTEGRATION.md snippets compiled against the reference headers
    (oracle/ref/integration_adapter.cpp)."""
    global _integ
    if _integ is None:
        ref()  # the reference library first (ref_init, its thread pool)
        L = C.CDLL(INTEG_SO)
        i8, u16, f32 = C.POINTER(C.c_int8), C.POINTER(C.c_uint16), C.POINTER(C.c_float)
        L.integ_mcf_u16.restype = C.c_int
        L.integ_mcf_u16.argtypes = [C.c_int] * 4 + [i8, C.c_uint16, C.c_uint16, u16,
                                                    C.POINTER(C.c_int), C.c_int, C.c_int, C.c_float]
        L.integ_mcf_f32.restype = C.c_int
        L.integ_mcf_f32.argtypes = [C.c_int] * 4 + [i8, C.c_float, C.c_float, f32,
                                                    C.POINTER(C.c_int), C.c_int, C.c_int, C.c_float,
                                                    C.c_int]
        L.integ_g2p_mr.restype = C.c_int
        L.integ_g2p_mr.argtypes = [C.c_void_p, C.c_void_p, C.c_int64, C.c_float]
        L.integ_splat.restype = C.c_int
        L.integ_splat.argtypes = [C.c_int] * 4 + [C.c_void_p, C.c_int64, C.c_int, C.c_float,
                                                  C.c_void_p, C.c_void_p]
        L.integ_pressure.restype = C.c_int
        L.integ_pressure.argtypes = [C.c_void_p] * 5 + [C.c_float, C.c_int, C.POINTER(C.c_int),
                                                        C.POINTER(C.c_int), C.POINTER(C.c_double)]
        _integ = L
    return _integ


def integ_mcf_u16(res3, bsx, kind, values, update, num_iter, dt, empty_val=0, full_val=65535):
    """INTEGRATION.md's render-density snippet on a reference grid; returns
    (status, values)."""
    L = integ()
    v = np.ascontiguousarray(values, np.uint16).copy()
    k = np.ascontiguousarray(kind, np.int8)
    u = np.ascontiguousarray(update, np.int32)
    rc = L.integ_mcf_u16(*res3, bsx, _p(k, C.c_int8), empty_val, full_val, _p(v, C.c_uint16),
                         _p(u, C.c_int), len(u), num_iter, dt)
    return rc, v


def integ_mcf_f32(res3, bsx, kind, values, update, num_iter, dt, clamp01=False, empty_val=4.0,
                  full_val=-4.0):
    """INTEGRATION.md's FP32 snippet on a reference grid; returns (status, values)."""
    L = integ()
    v = np.ascontiguousarray(values, np.float32).copy()
    k = np.ascontiguousarray(kind, np.int8)
    u = np.ascontiguousarray(update, np.int32)
    rc = L.integ_mcf_f32(*res3, bsx, _p(k, C.c_int8), empty_val, full_val, _p(v, C.c_float),
                         _p(u, C.c_int), len(u), num_iter, dt, int(bool(clamp01)))
    return rc, v


def integ_splat(res3, bsx, pos, num_iter, dt):
    """INTEGRATION.md's splat snippet on a reference grid without blocks;
    returns (status, active block flags, values of the active blocks)."""
    L = integ()
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    nb = (res3[0] // bsx) * (res3[1] // bsx) * (res3[2] // bsx)
    act = np.zeros(nb, np.int8)
    vals = np.zeros(nb * bsx ** 3, np.uint16)
    rc = L.integ_splat(*res3, bsx, p.ctypes.data, len(p), num_iter, dt, act.ctypes.data,
                       vals.ctypes.data)
    return rc, act, vals[: int(act.sum()) * bsx ** 3]


def integ_pressure(ref_handle, scene, tol, max_iter):
    """INTEGRATION.md's pressure snippet on a grid the reference prepared
    (ref_pressure.RefPressure.h); the solution lands in its CH_PRESSURE.
    Returns (status code, solve status, iterations, relative residual)."""
    L = integ()
    cb = scene.callbacks()
    st, it, rr = C.c_int(), C.c_int(), C.c_double()
    rc = L.integ_pressure(ref_handle, cb.sampleCellType, cb.sampleFaceCoeff, cb.sampleRhs,
                          cb.user, tol, max_iter, C.byref(st), C.byref(it), C.byref(rr))
    return rc, st.value, it.value, rr.value


def ref():
    global _ref
    if _ref is None:
        if not os.path.exists(REF_SO):
            raise FileNotFoundError(REF_SO)
        L = C.CDLL(REF_SO)
        L.ref_init.restype = C.c_int
        L.ref_init.argtypes = [C.c_int]
        L.ref_mcf.restype = C.c_int
        L.ref_mcf.argtypes = [C.c_int] * 4 + [C.POINTER(C.c_int8), C.c_float, C.c_float,
                                              C.POINTER(C.c_float), C.POINTER(C.c_int), C.c_int,
                                              C.c_int, C.c_float, C.c_int,
                                              C.POINTER(C.c_double)]
        L.ref_init(0)
        _ref = L
    return _ref


def mcf_oracle(nb3, bsx, kind, values, update, num_iter, dt, clamp01=False, empty_val=4.0,
               full_val=-4.0, exact_iter=False):
    """C restatement of the 8-colour MCF smoother; returns the new values."""
    nbx, nby, nbz = nb3
    v = np.ascontiguousarray(values, np.float32).copy()
    kind = np.ascontiguousarray(kind, np.int8)
    up = np.ascontiguousarray(update, np.int32)
    rc = oracle().oracle_mcf(nbx, nby, nbz, bsx, _p(kind, C.c_int8), empty_val, full_val,
                             _p(v, C.c_float), _p(up, C.c_int), len(up), num_iter, dt,
                             int(bool(clamp01)), int(bool(exact_iter)))
    if rc:
        raise RuntimeError(f"oracle_mcf rc={rc}")
    return v


def mcf_reference(res3, bsx, kind, values, update, num_iter, dt, clamp01=False, empty_val=4.0,
                  full_val=-4.0, threads=0):
    """Compiled reference applyChannelPdeFast<float>; returns (values, seconds)."""
    L = ref()
    if threads:
        L.ref_init(threads)
    sx, sy, sz = res3
    v = np.ascontiguousarray(values, np.float32).copy()
    kind = np.ascontiguousarray(kind, np.int8)
    up = np.ascontiguousarray(update, np.int32)
    secs = C.c_double(0)
    rc = L.ref_mcf(sx, sy, sz, bsx, _p(kind, C.c_int8), empty_val, full_val, _p(v, C.c_float),
                   _p(up, C.c_int), len(up), num_iter, dt, int(bool(clamp01)), C.byref(secs))
    if rc:
        raise RuntimeError(f"ref_mcf rc={rc}")
    return v, secs.value


def mcf_reference_u16(res3, bsx, kind, values, update, num_iter, dt, clamp01=True,
                      empty_val=0, full_val=65535):
    """Compiled reference applyChannelPdeFast<uint16_t> (16-bit render density,
    the reference's RenderDensity); values are raw 16-bit integers.  Returns
    (values, seconds)."""
    L = ref()
    if not hasattr(L, "_u16_sig"):
        L.ref_mcf_u16.restype = C.c_int
        L.ref_mcf_u16.argtypes = [C.c_int] * 4 + [C.POINTER(C.c_int8), C.c_uint16, C.c_uint16,
                                                  C.POINTER(C.c_uint16), C.POINTER(C.c_int),
                                                  C.c_int, C.c_int, C.c_float, C.c_int,
                                                  C.POINTER(C.c_double)]
        L._u16_sig = True
    sx, sy, sz = res3
    v = np.ascontiguousarray(values, np.uint16).copy()
    kind = np.ascontiguousarray(kind, np.int8)
    up = np.ascontiguousarray(update, np.int32)
    secs = C.c_double(0)
    rc = L.ref_mcf_u16(sx, sy, sz, bsx, _p(kind, C.c_int8), empty_val, full_val,
                       _p(v, C.c_uint16), _p(up, C.c_int), len(up), num_iter, dt,
                       int(bool(clamp01)), C.byref(secs))
    if rc:
        raise RuntimeError(f"ref_mcf_u16 rc={rc}")
    return v, secs.value


def pressure_oracle(scene, tol=1e-12, max_iter=20000, domain_bc=None):
    """FP64 CG solution of the pressure system of a msbg_gpu.PressureScene.

    Returns (x, b, iterations, true relative residual); x, b in the
    reference block layout.  domain_bc: six DBC values (0 open, 1 solid) or
    None for the reference's rule."""
    L = oracle()
    if not hasattr(L, "_ps_sig"):
        L.oracle_pressure_solve.restype = C.c_int
        L.oracle_pressure_solve.argtypes = [C.c_int] * 4 + [C.POINTER(C.c_int)] * 2 + [C.c_void_p] * 4 + [
            C.c_double, C.c_int, C.POINTER(C.c_double), C.POINTER(C.c_double),
            C.POINTER(C.c_int), C.POINTER(C.c_double)]
        L.oracle_pressure_apply.restype = C.c_int
        L.oracle_pressure_apply.argtypes = [C.c_int] * 4 + [C.POINTER(C.c_int)] * 2 + [C.c_void_p] * 3 + [
            C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L._ps_sig = True
    n = scene.packed_size()
    x = np.zeros(n, np.float64)
    b = np.zeros(n, np.float64)
    it = C.c_int()
    rr = C.c_double()
    cb = scene.callbacks()
    bl = np.ascontiguousarray(scene.block_levels, np.int32)
    dbc = None if domain_bc is None else np.ascontiguousarray(domain_bc, np.int32)
    rc = L.oracle_pressure_solve(scene.res, scene.res, scene.res, scene.bsx0, _p(bl, C.c_int),
                                 None if dbc is None else _p(dbc, C.c_int), cb.sampleCellType, cb.sampleFaceCoeff, cb.sampleRhs, cb.user,
                                 tol, max_iter, _p(x, C.c_double), _p(b, C.c_double),
                                 C.byref(it), C.byref(rr))
    if rc:
        raise RuntimeError(f"oracle_pressure_solve rc={rc}")
    return x, b, it.value, rr.value


def pressure_apply_oracle(scene, x, domain_bc=None):
    L = oracle()
    pressure_oracle  # signatures are set on first solve
    if not hasattr(L, "_ps_sig"):
        pressure_oracle(scene, tol=1.0, max_iter=0)
    cb = scene.callbacks()
    bl = np.ascontiguousarray(scene.block_levels, np.int32)
    xx = np.ascontiguousarray(x, np.float64)
    y = np.zeros_like(xx)
    dbc = None if domain_bc is None else np.ascontiguousarray(domain_bc, np.int32)
    rc = L.oracle_pressure_apply(scene.res, scene.res, scene.res, scene.bsx0, _p(bl, C.c_int),
                                 None if dbc is None else _p(dbc, C.c_int), cb.sampleCellType, cb.sampleFaceCoeff, cb.user,
                                 _p(xx, C.c_double), _p(y, C.c_double))
    if rc:
        raise RuntimeError(f"oracle_pressure_apply rc={rc}")
    return y


class ArrayScene:
    """Pressure problem given by per-cell arrays in the packed block layout of
    MG level 0 (flags, lower-face coefficients per direction, rhs), with the
    interface of msbg_gpu.PressureScene that the oracle functions read.  Its
    callbacks are C functions of the oracle library
    (oracle_array_scene_*, oracle/msbg_oracle_pressure.c)."""

    def __init__(self, res, bsx0, n_levels, block_levels, flags, face, rhs):
        L = oracle()
        if not hasattr(L, "_arr_sig"):
            L.oracle_array_scene_create.restype = C.c_void_p
            L.oracle_array_scene_create.argtypes = [C.c_int] * 4 + [
                C.POINTER(C.c_int), C.POINTER(C.c_uint16)] + [C.POINTER(C.c_float)] * 4
            L.oracle_array_scene_destroy.argtypes = [C.c_void_p]
            L._arr_sig = True
        self._L = L
        self.res, self.bsx0, self.n_levels = res, bsx0, n_levels
        self.block_levels = np.ascontiguousarray(block_levels, np.int32)
        self.flags = np.ascontiguousarray(flags, np.uint16)
        self.face = [np.ascontiguousarray(f, np.float32) for f in face]
        self.rhs = np.ascontiguousarray(rhs, np.float32)
        self.h = L.oracle_array_scene_create(res, res, res, bsx0, _p(self.block_levels, C.c_int),
                                             _p(self.flags, C.c_uint16),
                                             *[_p(f, C.c_float) for f in self.face],
                                             _p(self.rhs, C.c_float))
        if not self.h:
            raise MemoryError("oracle_array_scene_create")

    def callbacks(self):
        L = self._L

        class _Cb:
            pass
        cb = _Cb()
        cb.sampleCellType = C.cast(L.oracle_array_cell_type, C.c_void_p).value
        cb.sampleFaceCoeff = C.cast(L.oracle_array_face, C.c_void_p).value
        cb.sampleRhs = C.cast(L.oracle_array_rhs, C.c_void_p).value
        cb.user = self.h
        return cb

    def packed_size(self):
        return int(sum((self.bsx0 >> int(l)) ** 3 for l in self.block_levels))

    def close(self):
        if self.h:
            self._L.oracle_array_scene_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------------------
# FLIP transfers (oracle/msbg_oracle_flip.c)
# ---------------------------------------------------------------------------
class _FlipParams(C.Structure):
    _fields_ = [("rhoL", C.c_float), ("rhoG", C.c_float), ("massEps", C.c_float),
                ("betaMin", C.c_float), ("alphaPhi", C.c_float), ("particlesPerVoxel", C.c_int)]


def _flip_lib():
    L = oracle()
    if not hasattr(L, "_flip_sig"):
        vp, i32, f32 = C.c_void_p, C.c_int, C.c_float
        L.oracle_flip_p2g.restype = i32
        L.oracle_flip_p2g.argtypes = [i32] * 4 + [vp, C.c_int64, C.POINTER(_FlipParams), vp, vp,
                                                 vp, vp]
        L.oracle_flip_gravity.argtypes = [i32] * 4 + [vp, vp, vp, f32, f32, f32]
        L.oracle_flip_gradient.argtypes = [i32] * 4 + [vp, vp, vp, vp, f32, f32]
        L.oracle_flip_g2p.argtypes = [i32] * 4 + [vp, C.c_int64, vp, vp, f32]
        L._flip_sig = True
    return L


def flip_p2g(res, bsx, particles, rhoL=1000.0, rhoG=1.0, massEps=1e-5, betaMin=1e-6,
             alphaPhi=1.0, ppv=8):
    """FlipSimulation::particleToGrid restated on the CPU: (vel[3n], mass[n],
    beta[3n], active block flags)."""
    L = _flip_lib()
    n = res ** 3
    vel = np.zeros(3 * n, np.float32)
    mass = np.zeros(n, np.float32)
    beta = np.zeros(3 * n, np.float32)
    act = np.zeros((res // bsx) ** 3, np.uint8)
    prm = _FlipParams(rhoL, rhoG, massEps, betaMin, alphaPhi, ppv)
    p = np.ascontiguousarray(particles)
    rc = L.oracle_flip_p2g(res, res, res, bsx, p.ctypes.data, len(p), C.byref(prm),
                           vel.ctypes.data, mass.ctypes.data, beta.ctypes.data, act.ctypes.data)
    if rc:
        raise RuntimeError(f"oracle_flip_p2g rc={rc}")
    return vel, mass, beta, act


def flip_gravity(res, bsx, vel, mass, gravity, dt, massEps=1e-5):
    """applyGravity restated: (vel, velOld)."""
    L = _flip_lib()
    v = np.array(vel, np.float32)
    old = np.zeros_like(v)
    m = np.ascontiguousarray(mass, np.float32)
    L.oracle_flip_gravity(res, res, res, bsx, v.ctypes.data, old.ctypes.data, m.ctypes.data,
                          gravity, dt, massEps)
    return v, old


def flip_gradient(res, bsx, vel, mass, beta, pressure, dt, massEps=1e-5):
    """The pressure-gradient update restated: the new vel."""
    L = _flip_lib()
    v = np.array(vel, np.float32)
    args = [np.ascontiguousarray(a, np.float32) for a in (mass, beta, pressure)]
    L.oracle_flip_gradient(res, res, res, bsx, v.ctypes.data, *[a.ctypes.data for a in args],
                           dt, massEps)
    return v


def flip_g2p(res, bsx, particles, vel, velOld, alpha):
    """gridToParticle restated (level-0 interpolation): updated particles."""
    L = _flip_lib()
    p = np.array(particles)
    v, o = np.ascontiguousarray(vel, np.float32), np.ascontiguousarray(velOld, np.float32)
    L.oracle_flip_g2p(res, res, res, bsx, p.ctypes.data, len(p), v.ctypes.data, o.ctypes.data,
                      alpha)
    return p


# ---- particle splatting (msbg_oracle_splat.c; src/msbg_demo.cpp) ----

def _splat_lib():
    L = oracle()
    if not hasattr(L, "_splat_sig"):
        vp, i32, f32 = C.c_void_p, C.c_int, C.c_float
        L.oracle_splat_domain.argtypes = [i32] * 3 + [vp, vp]
        L.oracle_splat_mark.restype = i32
        L.oracle_splat_mark.argtypes = [i32] * 4 + [vp, C.c_int64, f32, f32, vp]
        L.oracle_splat.restype = i32
        L.oracle_splat.argtypes = [i32] * 4 + [vp, vp, C.c_int64, f32, f32, i32, vp]
        L.oracle_splat_finalize_value.restype = C.c_uint16
        L.oracle_splat_finalize_value.argtypes = [C.c_uint16, f32, f32]
        L._splat_sig = True
    return L


def splat_domain(res3):
    """The demo's particle domain bounds (lo[3], hi[3]) restated."""
    L = _splat_lib()
    lo = np.zeros(3, np.float32)
    hi = np.zeros(3, np.float32)
    L.oracle_splat_domain(*res3, lo.ctypes.data, hi.ctypes.data)
    return lo, hi


def splat_mark(res3, bsx, pos, r_particle=2.0, nb_dist=2.0):
    """Active-block marking restated: one byte per block (1 = active)."""
    L = _splat_lib()
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    nb = (res3[0] // bsx) * (res3[1] // bsx) * (res3[2] // bsx)
    act = np.zeros(nb, np.int8)
    rc = L.oracle_splat_mark(*res3, bsx, p.ctypes.data, len(p), r_particle, nb_dist,
                             act.ctypes.data)
    if rc:
        raise RuntimeError(f"oracle_splat_mark rc={rc}")
    return act


def splat(res3, bsx, kind, pos, r_particle=2.0, nb_dist=2.0, finalize=True):
    """The splat restated: the value blocks (kind == 1) packed in bid order."""
    L = _splat_lib()
    p = np.ascontiguousarray(pos, np.float32).reshape(-1, 3)
    k = np.ascontiguousarray(kind, np.int8)
    out = np.zeros(int((k == 1).sum()) * bsx ** 3, np.uint16)
    rc = L.oracle_splat(*res3, bsx, k.ctypes.data, p.ctypes.data, len(p), r_particle, nb_dist,
                        1 if finalize else 0, out.ctypes.data)
    if rc:
        raise RuntimeError(f"oracle_splat rc={rc}")
    return out


def splat_finalize_table(r_particle=2.0, nb_dist=2.0):
    """The finalisation of every 16-bit squared distance (65536 entries)."""
    L = _splat_lib()
    return np.array([L.oracle_splat_finalize_value(q, r_particle, nb_dist) for q in range(65536)],
                    np.uint16)


SPLAT_REF_SO = os.path.join(OUT, "libmsbg_splatref.so")
_splat_ref = None


def splat_reference_available():
    return os.path.exists(SPLAT_REF_SO) and os.path.exists(REF_SO)


def _splat_ref_lib():
    global _splat_ref
    if _splat_ref is None:
        ref()  # the reference library first (ref_init, its thread pool)
        L = C.CDLL(SPLAT_REF_SO)
        L.ref_splat_demo.restype = C.c_int
        L.ref_splat_demo.argtypes = [C.c_int, C.c_char_p] + [C.c_int] * 4
        L.ref_splat_sizes.argtypes = [C.c_void_p]
        L.ref_splat_copy.argtypes = [C.c_void_p] * 5
        L.ref_splat_times.argtypes = [C.c_void_p]
        L.ref_splat_in_domain.restype = C.c_int
        L.ref_splat_in_domain.argtypes = [C.c_int] * 4 + [C.c_void_p, C.c_int64, C.c_void_p]
        _splat_ref = L
    return _splat_ref


def write_ply(path, points):
    """An ASCII PLY with the vertices the demo's reader takes
    (readVerticesFromPLY, src/msbg_demo.cpp:72-120)."""
    with open(path, "w") as f:
        f.write("ply\nformat ascii 1.0\nelement vertex %d\n" % len(points))
        f.write("property float x\nproperty float y\nproperty float z\nend_header\n")
        for p in points:
            f.write("%.6f %.6f %.6f\n" % (p[0], p[1], p[2]))


def splat_reference_demo(ply_path, test_case, bsx, res3):
    """Runs the reference's msbg_test_sparse on a PLY file up to its
    smoothing call (oracle/ref/splat_harness.cpp) and returns what it
    splatted: particle positions, the value blocks, the quantised squared
    distances after the splat loop, the render density after finalisation,
    and the phase times."""
    L = _splat_ref_lib()
    rc = L.ref_splat_demo(test_case, ply_path.encode(), bsx, *res3)
    if rc:
        raise RuntimeError(f"ref_splat_demo rc={rc}")
    sz = np.zeros(5, np.int64)
    L.ref_splat_sizes(sz.ctypes.data)
    n, nr, nf, b, _ = (int(v) for v in sz)
    pos = np.zeros((n, 3), np.float32)
    rb = np.zeros(nr, np.int32)
    raw = np.zeros(nr * b ** 3, np.uint16)
    fb = np.zeros(nf, np.int32)
    fv = np.zeros(nr * b ** 3, np.uint16)
    L.ref_splat_copy(pos.ctypes.data, rb.ctypes.data, raw.ctypes.data, fb.ctypes.data,
                     fv.ctypes.data)
    t = np.zeros(3, np.float64)
    L.ref_splat_times(t.ctypes.data)
    return {"pos": pos, "blocks": rb, "raw": raw, "active": fb, "final": fv, "bsx": b,
            "t_marked": t[0], "t_splat": t[1], "t_final": t[2]}


def splat_reference_in_domain(res3, bsx, pts):
    """The demo's particle test run by the reference on a grid it creates."""
    L = _splat_ref_lib()
    p = np.ascontiguousarray(pts, np.float32).reshape(-1, 3)
    out = np.zeros(len(p), np.int32)
    rc = L.ref_splat_in_domain(*res3, bsx, p.ctypes.data, len(p), out.ctypes.data)
    if rc:
        raise RuntimeError(f"ref_splat_in_domain rc={rc}")
    return out


# ---- mixed-resolution G2P interpolation (msbg_oracle_flip_mr.c) ----

def _mr_lib():
    L = oracle()
    if not hasattr(L, "_mr_sig"):
        vp, i32, f32 = C.c_void_p, C.c_int, C.c_float
        L.oracle_mr_layout.restype = C.c_int64
        L.oracle_mr_layout.argtypes = [i32] * 4 + [vp, vp]
        L.oracle_mr_dist.argtypes = [i32] * 4 + [vp, i32, i32, vp, vp]
        L.oracle_mr_dist_interp.argtypes = [i32] * 7 + [vp, vp, vp, vp, i32, i32, vp, C.c_int64,
                                                        vp]
        L.oracle_mr_g2p.argtypes = [i32] * 4 + [vp, i32, vp, C.c_int64, vp, vp, vp, vp, f32]
        L.oracle_mr_downsample_velocity.argtypes = [i32] * 4 + [vp, i32, vp, vp, vp]
        L._mr_sig = True
    return L


def mr_layout(nb3, bsx0, level):
    """Packed layout of a mixed-resolution grid: (first voxel per block, total)."""
    L = _mr_lib()
    lv = np.ascontiguousarray(level, np.int32)
    off = np.zeros(lv.size, np.int64)
    n = L.oracle_mr_layout(nb3[0], nb3[1], nb3[2], bsx0, lv.ctypes.data, off.ctypes.data)
    return off, int(n)


def mr_dist(nb3, bsx0, level, n_levels, dtrans=6):
    """CH_DIST_FINECOARSE restated: (packed uint16 distances of the value
    blocks, block kinds per level [n_levels, nBlocks]: 0 empty, 1 value, 2 full)."""
    L = _mr_lib()
    lv = np.ascontiguousarray(level, np.int32)
    _, n = mr_layout(nb3, bsx0, lv)
    dist = np.zeros(n, np.uint16)
    kind = np.zeros((n_levels, lv.size), np.int8)
    L.oracle_mr_dist(nb3[0], nb3[1], nb3[2], bsx0, lv.ctypes.data, n_levels, dtrans,
                     dist.ctypes.data, kind.ctypes.data)
    return dist, kind


def mr_dist_interp(res3, bsx0, level, dist, kind, lv, pos, dtrans=6):
    """The distance channel of level lv interpolated at pos (level units, n x 3)."""
    L = _mr_lib()
    nb3 = [r // bsx0 for r in res3]
    lev = np.ascontiguousarray(level, np.int32)
    off, _ = mr_layout(nb3, bsx0, lev)
    p = np.ascontiguousarray(pos, np.float32)
    out = np.zeros(len(p), np.float32)
    L.oracle_mr_dist_interp(res3[0], res3[1], res3[2], bsx0, *nb3, lev.ctypes.data,
                            off.ctypes.data, np.ascontiguousarray(dist, np.uint16).ctypes.data,
                            np.ascontiguousarray(kind, np.int8).ctypes.data, dtrans, lv,
                            p.ctypes.data, len(p), out.ctypes.data)
    return out


def mr_g2p(res3, bsx0, level, particles, vel, velOld, dist, kind, alpha, dtrans=6):
    """gridToParticle through interpVec3MSBG restated: updated particles."""
    L = _mr_lib()
    lev = np.ascontiguousarray(level, np.int32)
    p = np.array(particles)
    v, o = np.ascontiguousarray(vel, np.float32), np.ascontiguousarray(velOld, np.float32)
    d = np.ascontiguousarray(dist, np.uint16)
    k = np.ascontiguousarray(kind, np.int8)
    L.oracle_mr_g2p(res3[0], res3[1], res3[2], bsx0, lev.ctypes.data, dtrans, p.ctypes.data,
                    len(p), v.ctypes.data, o.ctypes.data, d.ctypes.data, k.ctypes.data, alpha)
    return p


def mg_levels(level0, m):
    """Block levels at MG level m: max(level0, m) (src/msbg.h:3574-3590)."""
    return np.maximum(np.asarray(level0, np.int32), m).astype(np.int32)


def mr_downsample_velocity(res3, bsx0, level0, m, flags, src):
    """downsampleVelocity restated: MG level m-1 (src, packed, 3 floats per
    voxel) to MG level m, with the MG-level-m cell flags; returns dst."""
    L = _mr_lib()
    lev = np.ascontiguousarray(level0, np.int32)
    _, n = mr_layout([r // bsx0 for r in res3], bsx0, mg_levels(lev, m))
    dst = np.zeros(3 * n, np.float32)
    L.oracle_mr_downsample_velocity(res3[0], res3[1], res3[2], bsx0, lev.ctypes.data, m,
                                    np.ascontiguousarray(flags, np.uint16).ctypes.data,
                                    np.ascontiguousarray(src, np.float32).ctypes.data,
                                    dst.ctypes.data)
    return dst


def _ref_mr():
    L = ref()
    if not hasattr(L, "_mr_sig"):
        vp = C.c_void_p
        L.ref_mr_create.restype = vp
        L.ref_mr_create.argtypes = [C.c_int] * 5 + [vp]
        L.ref_mr_destroy.argtypes = [vp]
        L.ref_mr_dtransres.restype = C.c_int
        L.ref_mr_dtransres.argtypes = [vp]
        L.ref_mr_block_info.argtypes = [vp, vp, vp]
        L.ref_mr_dist.restype = C.c_longlong
        L.ref_mr_dist.argtypes = [vp, vp, vp]
        L.ref_mr_dist_interp.argtypes = [vp, C.c_int, vp, C.c_longlong, vp]
        L.ref_mr_set_vec.restype = C.c_int
        L.ref_mr_set_vec.argtypes = [vp, C.c_int, vp]
        L._mr_sig = True
    return L


class RefMultires:
    """A reference MultiresSparseGrid with the given block levels, set up by its
    own setRefinementMap (which builds the fine/coarse distance channel)."""

    def __init__(self, res3, bsx0, n_levels, level):
        self.L = _ref_mr()
        self.level = np.ascontiguousarray(level, np.int32)
        self.h = self.L.ref_mr_create(res3[0], res3[1], res3[2], bsx0, n_levels,
                                      self.level.ctypes.data)
        if not self.h:
            raise RuntimeError("ref_mr_create failed")
        self.nb3 = [r // bsx0 for r in res3]
        self.bsx0 = bsx0

    def dtrans(self):
        return self.L.ref_mr_dtransres(self.h)

    def block_info(self):
        lv = np.zeros(self.level.size, np.int32)
        fl = np.zeros(self.level.size, np.int32)
        self.L.ref_mr_block_info(self.h, lv.ctypes.data, fl.ctypes.data)
        return lv, fl

    def dist(self, n_levels):
        _, n = mr_layout(self.nb3, self.bsx0, self.level)
        out = np.zeros(n, np.uint16)
        kind = np.zeros((n_levels, self.level.size), np.int8)
        got = self.L.ref_mr_dist(self.h, out.ctypes.data, kind.ctypes.data)
        if got != n:
            raise RuntimeError(f"ref_mr_dist returned {got}, packed size {n}")
        return out, kind

    def dist_interp(self, lv, pos):
        p = np.ascontiguousarray(pos, np.float32)
        out = np.zeros(len(p), np.float32)
        self.L.ref_mr_dist_interp(self.h, lv, p.ctypes.data, len(p), out.ctypes.data)
        return out

    def set_vec(self, ch, packed):
        """Fills vector channel ch of every level from the packed layout."""
        d = np.ascontiguousarray(packed, np.float32)
        if self.L.ref_mr_set_vec(self.h, ch, d.ctypes.data):
            raise RuntimeError("ref_mr_set_vec failed")

    def close(self):
        if self.h:
            self.L.ref_mr_destroy(self.h)
            self.h = None
