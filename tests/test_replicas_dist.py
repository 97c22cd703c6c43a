"""The multi-GPU bench path on CPU: `bench.py --gpus N` runs N independent
replicas of the solve (the pressure solve has no data-path exchange), joined
only by a barrier and the max-over-ranks timing.  Here two gloo ranks check
that plumbing and that replicas of the host-side problem build agree."""
import os

import pytest
import torch.multiprocessing as mp


def _rank(rank, ws, port, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    import bench
    import msbg_gpu
    ws_, rank_, _ = bench.dist_env()
    dist = bench.init_dist(ws_, backend="gloo")
    # each replica builds the same problem on the host
    s = msbg_gpu.PressureScene(64, 16, 2, band=4.0, seed=21)
    fluid = msbg_gpu.count_liquid_cells(s)
    dist.barrier()
    # max over ranks of a per-rank time, as the bench reports it
    t = bench.max_over_ranks(dist, 1.0 + rank_, "cpu")
    f = bench.max_over_ranks(dist, float(fluid), "cpu")
    q.put((rank_, t, fluid, f))
    dist.barrier()
    dist.destroy_process_group()


def test_two_gloo_replicas_barrier_and_max_over_ranks():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 29500 + os.getpid() % 1000
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = sorted(q.get(timeout=240) for _ in range(2))
    for p in ps:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert [o[0] for o in out] == [0, 1]
    assert all(o[1] == 2.0 for o in out)          # max over ranks of 1.0 and 2.0
    assert out[0][2] == out[1][2] == out[0][3]    # identical replicas


def _failing_rank(rank, ws, port, q):
    """Rank 1 raises before its first collective (a replica that failed on
    the host); rank 0 must end its barrier with an error, not wait."""
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(ws), LOCAL_RANK=str(rank))
    import time

    import bench
    dist = bench.init_dist(ws, backend="gloo", timeout_s=5)
    if rank == 1:
        q.put((1, "raised"))
        raise SystemExit(3)
    t0 = time.perf_counter()
    try:
        dist.barrier()
        bench.max_over_ranks(dist, 1.0, "cpu")
        q.put((0, "no error"))
    except Exception as e:  # the failed peer ends the collective
        q.put((0, f"error after {time.perf_counter() - t0:.1f} s: {type(e).__name__}"))


def test_failed_replica_ends_the_others_collective_with_an_error():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = 30500 + os.getpid() % 1000
    ps = [ctx.Process(target=_failing_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    out = dict(q.get(timeout=120) for _ in range(2))
    for p in ps:
        p.join(timeout=60)
    assert ps[1].exitcode == 3
    assert out[0].startswith("error after"), out[0]
    assert float(out[0].split()[2]) < 30.0
