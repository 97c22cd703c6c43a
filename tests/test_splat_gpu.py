"""GPU particle splatting (csrc/splat.cu) against the reference and the oracle.

- The reference's own demo output (tests/golden/splat_*.npz, made by running
  msbg_test_sparse of src/msbg_demo.cpp, tests/golden/make_splat_golden.py):
  the GPU must reproduce its value blocks, its quantised squared distances
  and its render density exactly.
- The pinned CPU restatement (oracle/msbg_oracle_splat.c) on larger seeded
  clouds, on caller-given block kinds (scans that stop at blocks without
  values), and on the edge cases: no particles, particles outside the domain,
  at its bounds, not finite.
- The splat feeds the smoother: the GPU splat followed by the GPU MCF equals
  the reference's MCF on the reference's splat within the 16-bit smoother's
  one-quantum tolerance.
"""
import os

import numpy as np
import pytest
import torch

import msbg_gpu
import oracle

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["splat_demo_b8", "splat_demo_b16", "splat_demo_b32"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, name + ".npz")))


def gpu_splat(res3, bsx, pos, kind=None, raw=False, r_particle=2.0, nb_dist=2.0, chan=3):
    ctx = msbg_gpu.Context(0)
    try:
        ctx.set_topology(*res3, bsx)
        k = ctx.splat(chan, pos, r_particle, nb_dist, kind=kind, raw=raw)
        out = np.empty(int((k == 1).sum()) * bsx ** 3, np.uint16)
        if len(out):
            ctx.download_channel_u16(chan, out)
        return k, out
    finally:
        ctx.close()


@pytest.mark.parametrize("name", CASES)
def test_gpu_reproduces_reference_demo(name):
    g = load(name)
    res3, bsx = tuple(int(v) for v in g["res"]), int(g["bsx"])
    k, fin = gpu_splat(res3, bsx, g["pos"])
    assert np.array_equal(np.nonzero(k == 1)[0], g["blocks"])
    assert set(np.unique(k)) <= {1, 2}
    assert np.array_equal(fin, g["final"])
    _, raw = gpu_splat(res3, bsx, g["pos"], raw=True)
    assert np.array_equal(raw, g["raw"])


@pytest.mark.parametrize("bsx,res,n_base,tc", [(8, 128, 64, 1), (16, 256, 96, 1),
                                               (32, 256, 64, 2), (16, 192, 48, 2)])
def test_gpu_matches_oracle_on_demo_clouds(bsx, res, n_base, tc):
    res3 = (res, res, res)
    pos = msbg_gpu.splat_demo_particles(res3, n_base, seed=bsx + res, test_case=tc)
    k, fin = gpu_splat(res3, bsx, pos)
    act = oracle.splat_mark(res3, bsx, pos)
    assert np.array_equal(k == 1, act == 1)
    assert np.array_equal(fin, oracle.splat(res3, bsx, act, pos))


def test_gpu_matches_oracle_dense_uniform():
    """Many particles per voxel: every bin long, heavy overlap."""
    res3, bsx = (64, 96, 128), 16
    rng = np.random.default_rng(5)
    pos = (rng.random((300000, 3)) * np.array([40, 60, 50]) + np.array([12, 20, 40]))
    pos = pos.astype(np.float32)
    k, fin = gpu_splat(res3, bsx, pos)
    act = oracle.splat_mark(res3, bsx, pos)
    assert np.array_equal(k == 1, act == 1)
    assert np.array_equal(fin, oracle.splat(res3, bsx, act, pos))
    _, raw = gpu_splat(res3, bsx, pos, raw=True)
    assert np.array_equal(raw, oracle.splat(res3, bsx, act, pos, finalize=False))


@pytest.mark.parametrize("bsx", [8, 16])
def test_gpu_caller_kinds_stop_scans(bsx):
    """Caller-given kinds with const and absent blocks among the value blocks:
    particles in blocks without values splat nothing; scans that meet such a
    block stop there."""
    res3 = (64, 64, 64)
    nb = (64 // bsx) ** 3
    rng = np.random.default_rng(bsx)
    kind = rng.choice(np.array([0, 1, 1, 1, 2, 3], np.int8), nb)
    pos = (rng.random((40000, 3)) * 63.9 + 0.05).astype(np.float32)
    k, raw = gpu_splat(res3, bsx, pos, kind=kind, raw=True)
    assert np.array_equal(k, kind)
    want = oracle.splat(res3, bsx, kind, pos, finalize=False)
    assert np.array_equal(raw, want)
    # the stop changed something: the same particles over all-value blocks reach more
    full = oracle.splat(res3, bsx, np.ones(nb, np.int8), pos, finalize=False)
    keep = np.repeat(kind == 1, bsx ** 3)
    assert (full[keep] < raw).any()


def test_gpu_edge_cases():
    res3, bsx = (32, 32, 48), 8
    lo, hi = oracle.splat_domain(res3)
    nxt = lambda x, d: np.nextafter(np.float32(x), np.float32(d), dtype=np.float32)  # noqa: E731
    pos = np.array([[lo[0], 5, 5], [nxt(lo[0], -1), 6, 6], [hi[0], 7, 7], [nxt(hi[0], 99), 8, 8],
                    [5, 5, hi[2]], [np.nan, 9, 9], [9, np.inf, 9], [-3, 4, 4], [40, 4, 4],
                    [16, 16, 24], [31.5, 31.5, 47.5]], np.float32)
    k, fin = gpu_splat(res3, bsx, pos)
    act = oracle.splat_mark(res3, bsx, pos)
    assert np.array_equal(k == 1, act == 1)
    assert np.array_equal(fin, oracle.splat(res3, bsx, act, pos))
    # no particles at all, and only dropped ones: no value blocks
    for p in (np.zeros((0, 3), np.float32), pos[[1, 3, 5, 6, 7, 8]]):
        k, fin = gpu_splat(res3, bsx, p)
        assert (k == 2).all() and len(fin) == 0


def test_gpu_rejects_bad_parameters():
    ctx = msbg_gpu.Context(0)
    try:
        ctx.set_topology(32, 32, 32, 8)
        pos = np.full((4, 3), 10.0, np.float32)
        with pytest.raises(msbg_gpu.MsbgError):  # reaches past the neighbouring blocks
            ctx.splat(1, pos, 4.0, 4.0)
        with pytest.raises(msbg_gpu.MsbgError):
            ctx.splat(1, pos, -1.0, 2.0)
        with pytest.raises(msbg_gpu.MsbgError):
            ctx.splat(1, pos, 2.0, 2.0, kind=np.full(64, 7, np.int8))
        ctx.splat(1, pos, 2.0, 2.0)  # the context still works
    finally:
        ctx.close()


def test_device_entry_equals_host_entry():
    res3, bsx = (128, 128, 128), 16
    pos = msbg_gpu.splat_demo_particles(res3, 80, seed=9)
    k_host, fin_host = gpu_splat(res3, bsx, pos)
    ctx = msbg_gpu.Context(0)
    try:
        ctx.set_topology(*res3, bsx)
        t = torch.from_numpy(pos).cuda()
        torch.cuda.synchronize()
        k = ctx.splat_device(4, t.data_ptr(), len(pos))
        out = np.empty_like(fin_host)
        ctx.download_channel_u16(4, out)
    finally:
        ctx.close()
    assert np.array_equal(k, k_host) and np.array_equal(out, fin_host)


@pytest.mark.skipif(not oracle.ref_available(), reason="reference not built")
def test_splat_then_smoother_matches_reference_pipeline():
    """The demo's pipeline (src/msbg_demo.cpp:519-727): splat, then
    applyChannelPdeFast<uint16_t> with 5 iterations (run as 6), dt 0.05 and
    the [0,1] clamp on the active blocks."""
    g = load("splat_demo_b16")
    res3, bsx = tuple(int(v) for v in g["res"]), int(g["bsx"])
    nb = (res3[0] // bsx) * (res3[1] // bsx) * (res3[2] // bsx)
    kind = np.full(nb, 2, np.int8)
    kind[g["blocks"]] = 1
    ref, _ = oracle.mcf_reference_u16(res3, bsx, kind, g["final"], g["blocks"], 5, 0.05,
                                      clamp01=True, empty_val=0, full_val=65535)
    ctx = msbg_gpu.Context(0)
    try:
        ctx.set_topology(*res3, bsx)
        k = ctx.splat(6, g["pos"])
        ctx.apply_channel_pde_mcf(6, np.nonzero(k == 1)[0].astype(np.int32), 5, 0.05,
                                  clamp01=True)
        got = ctx.download_channel_u16(6, np.empty_like(g["final"]))
    finally:
        ctx.close()
    d = np.abs(got.astype(np.int64) - ref.astype(np.int64))
    assert (ref != g["final"]).any()
    assert d.max() <= 2 and (d > 0).mean() <= 2e-3, (int(d.max()), float((d > 0).mean()))
