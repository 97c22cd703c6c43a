"""The smoother entry point that allocates nothing (msbg_gpu_pde_mcf_noalloc).

It serves callers that cannot let the library allocate device memory: codes
that reserve all device memory with their own pool allocator, and threads
that must not block in the CUDA allocator during a time step.  Its only
scratch is a fixed device array inside the library.  This test is the
caller: it owns the device buffers (allocated with torch) and checks that
two calls in a row give what the context-based entry point gives, within the
smoother's FP32 parity tolerance.  The file is named to be collected last.
"""
import ctypes as C

import numpy as np
import pytest

import msbg_gpu

pytestmark = pytest.mark.gpu


def _fn():
    L = msbg_gpu.lib()
    f = L.msbg_gpu_pde_mcf_noalloc
    f.restype = C.c_int
    f.argtypes = [C.c_void_p, C.c_void_p, C.POINTER(C.c_int), C.c_int, C.c_int, C.c_int, C.c_int,
                  C.c_int, C.c_float, C.c_float, C.c_int, C.c_float, C.c_int, C.c_void_p,
                  C.POINTER(C.c_int)]
    return f


def tol_ok(a, b, rel=1e-5):
    return float((np.abs(a - b) / np.maximum(1.0, np.abs(b))).max()) <= rel


@pytest.mark.parametrize("bsx", [8, 16])
def test_noalloc_matches_context_entry_point_on_two_calls(bsx):
    import torch

    res = 128
    kind, vals = msbg_gpu.sphere_sdf_scene(res, bsx, n_spheres=10, rmin=10, rmax=30, seed=77)
    kind = kind.copy()
    kind[np.nonzero(kind == 2)[0][::3]] = 0  # some NULL blocks: Neumann halo
    vals = vals[: int((kind == 1).sum())]
    upd = np.nonzero(kind == 1)[0].astype(np.int32)
    upd = np.ascontiguousarray(upd[::-1])  # any order: the entry point regroups by colour
    nb1 = res // bsx

    # reference path: the context-based entry point, two calls of 2 iterations
    ctx = msbg_gpu.Context(0)
    ctx.set_topology(res, res, res, bsx)
    ctx.upload_channel(3, 0, kind, vals, 4.0, -4.0)
    expect = []
    for _ in range(2):
        ctx.apply_channel_pde_mcf(3, upd, 2, 0.1)
        expect.append(ctx.download_channel(3, np.empty_like(vals)))
    ctx.close()

    # no-allocation path: caller-owned device buffers, caller stream
    slot = np.where(kind == 1, np.cumsum(kind == 1) - 1,
                    np.where(kind == 2, -2, np.where(kind == 3, -3, -1))).astype(np.int32)
    dev = torch.device("cuda", 0)
    pool = torch.from_numpy(vals.copy()).to(dev)
    slot_t = torch.from_numpy(slot).to(dev)
    stream = torch.cuda.current_stream()
    f = _fn()
    timed_out = C.c_int(-1)
    for call in range(2):
        rc = f(C.c_void_p(pool.data_ptr()), C.c_void_p(slot_t.data_ptr()),
               upd.ctypes.data_as(C.POINTER(C.c_int)), len(upd), nb1, nb1, nb1, bsx, 4.0, -4.0, 2,
               0.1, 0, C.c_void_p(stream.cuda_stream), C.byref(timed_out))
        assert rc == 0, rc
        assert timed_out.value == 0
        got = pool.cpu().numpy()
        assert tol_ok(got, expect[call]), call


def test_noalloc_rejects_too_many_blocks_and_bad_ids():
    import torch

    f = _fn()
    dev = torch.device("cuda", 0)
    pool = torch.zeros(8 * 8 ** 3, device=dev)
    slot = torch.arange(8, dtype=torch.int32, device=dev)
    too_many = np.zeros(262144 + 1, np.int32)
    rc = f(C.c_void_p(pool.data_ptr()), C.c_void_p(slot.data_ptr()),
           too_many.ctypes.data_as(C.POINTER(C.c_int)), len(too_many), 2, 2, 2, 8, 0.0, 0.0, 2,
           0.1, 0, None, None)
    assert rc == 5
    bad = np.array([8], np.int32)  # block id outside the 2x2x2 raster
    rc = f(C.c_void_p(pool.data_ptr()), C.c_void_p(slot.data_ptr()),
           bad.ctypes.data_as(C.POINTER(C.c_int)), 1, 2, 2, 2, 8, 0.0, 0.0, 2, 0.1, 0, None, None)
    assert rc == 5
