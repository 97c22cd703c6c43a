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


def _scene(res, bsx):
    kind, vals = msbg_gpu.sphere_sdf_scene(res, bsx, n_spheres=10, rmin=10, rmax=30, seed=77)
    kind = kind.copy()
    kind[np.nonzero(kind == 2)[0][::3]] = 0  # some NULL blocks: Neumann halo
    vals = vals[: int((kind == 1).sum())]
    upd = np.nonzero(kind == 1)[0].astype(np.int32)
    upd = np.ascontiguousarray(upd[::-1])  # any order: the entry point regroups by colour
    slot = np.where(kind == 1, np.cumsum(kind == 1) - 1,
                    np.where(kind == 2, -2, np.where(kind == 3, -3, -1))).astype(np.int32)
    return kind, vals, upd, slot


def _context_result(res, bsx, kind, vals, upd, clamp01, calls):
    ctx = msbg_gpu.Context(0)
    ctx.set_topology(res, res, res, bsx)
    ctx.upload_channel(3, 0, kind, vals, 4.0, -4.0)
    expect = []
    for _ in range(calls):
        ctx.apply_channel_pde_mcf(3, upd, 2, 0.1, clamp01=clamp01)
        expect.append(ctx.download_channel(3, np.empty_like(vals)))
    ctx.close()
    return expect


def _call(f, pool, slot_t, lst, nb1, bsx, clamp01, stream, timed_out):
    return f(C.c_void_p(pool.data_ptr()), C.c_void_p(slot_t.data_ptr()),
             lst.ctypes.data_as(C.POINTER(C.c_int)), len(lst), nb1, nb1, nb1, bsx, 4.0, -4.0, 2,
             0.1, clamp01, C.c_void_p(stream.cuda_stream), C.byref(timed_out))


@pytest.mark.parametrize("bsx,clamp01", [(8, 0), (16, 0), (16, 1), (32, 0), (32, 1)])
def test_noalloc_matches_context_entry_point_on_two_calls(bsx, clamp01):
    import torch

    res = 128
    kind, vals, upd, slot = _scene(res, bsx)
    nb1 = res // bsx
    # reference path: the context-based entry point, two calls of 2 iterations
    expect = _context_result(res, bsx, kind, vals, upd, clamp01, 2)

    # no-allocation path: caller-owned device buffers, caller stream
    dev = torch.device("cuda", 0)
    pool = torch.from_numpy(vals.copy()).to(dev)
    slot_t = torch.from_numpy(slot).to(dev)
    stream = torch.cuda.current_stream()
    f = _fn()
    timed_out = C.c_int(-1)
    for call in range(2):
        torch.cuda.synchronize()
        free0 = torch.cuda.mem_get_info(0)[0]
        rc = _call(f, pool, slot_t, upd, nb1, bsx, clamp01, stream, timed_out)
        torch.cuda.synchronize()
        free1 = torch.cuda.mem_get_info(0)[0]
        assert rc == 0, rc
        assert timed_out.value == 0
        if call == 1:  # after the first call has loaded the module: no device memory taken
            assert free1 == free0, (free0, free1)
        got = pool.cpu().numpy()
        assert tol_ok(got, expect[call]), call


def test_noalloc_skips_and_reports_listed_non_value_blocks():
    """A const or NULL block id in the list is skipped on the device (nothing is
    written before the pool) and the call reports MSBG_EINVARG; the listed value
    blocks are still smoothed exactly as without the bad id."""
    import torch

    res, bsx = 128, 16
    kind, vals, upd, slot = _scene(res, bsx)
    nb1 = res // bsx
    expect = _context_result(res, bsx, kind, vals, upd, 0, 1)[0]
    bad_ids = [int(np.nonzero(kind == 2)[0][0]), int(np.nonzero(kind == 0)[0][0])]
    lst = np.ascontiguousarray(np.concatenate([upd, np.array(bad_ids, np.int32)]))
    dev = torch.device("cuda", 0)
    guard = 4096
    buf = torch.full((guard + vals.size + guard,), 7.0, device=dev)  # guard zones around the pool
    buf[guard:guard + vals.size] = torch.from_numpy(vals.ravel()).to(dev)
    pool = buf[guard:guard + vals.size]
    slot_t = torch.from_numpy(slot).to(dev)
    stream = torch.cuda.current_stream()
    timed_out = C.c_int(-1)
    rc = _call(_fn(), pool, slot_t, lst, nb1, bsx, 0, stream, timed_out)
    assert rc == 5, rc
    assert timed_out.value == 0
    host = buf.cpu().numpy()
    assert (host[:guard] == 7.0).all() and (host[-guard:] == 7.0).all()
    assert tol_ok(host[guard:guard + vals.size].reshape(vals.shape), expect)


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
