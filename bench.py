#!/usr/bin/env python
"""Benchmark of the B200 sparse block-grid solver.

Workload ``mcf`` (smoother at the 512^3 sphere-band configuration): one step =
one MultiresSparseGrid::applyChannelPdeFast-equivalent call, i.e. 20
iterations x 8 colour passes of the mean-curvature-flow smoother over every
value block (512^3, 16^3 blocks, band +-4 around 64 seeded spheres,
dt = 0.1), data resident in HBM.

Prints one JSON line (rank 0).  ``--impl reference`` times the reference's own
CPU implementation instead (compiled from the reference sources into
oracle/_ref/libmsbg_ref.so) on the same configuration.

Multi-GPU: the smoother runs as independent replicas, one per rank (no data
path collective); value = all ranks' voxel updates / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "msbg-flip_b200"))

METRIC = "MGPCG time-to-1e-6 & Gvoxel/s/iter: learned+mixed vs plain FP32, one B200"

MCF_CFG = dict(res=512, bsx=16, n_spheres=64, rmin=20.0, rmax=60.0, band=4.0, dilate=1,
               seed=1234, iters=20, dt=0.1)


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


class Clocks:
    """Samples nvidia-smi clocks during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.25)
        return self

    def __exit__(self, *a):
        if self.p:
            self.p.terminate()
            try:
                self.p.wait(5)
            except Exception:
                self.p.kill()

    def summary(self):
        self.f.flush()
        self.f.seek(0)
        mhz, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                mhz.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(mhz) if mhz else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(mhz)}


def read_traffic(name):
    """Per-cell DRAM traffic of a kernel from its committed ncu summary."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith("dram_bytes_per_cell="):
            return float(line.split("=")[1])
    return None


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def mcf_scene():
    import msbg_gpu
    c = MCF_CFG
    kind, vals = msbg_gpu.sphere_sdf_scene(c["res"], c["bsx"], c["n_spheres"], c["rmin"], c["rmax"],
                                           c["band"], c["dilate"], c["seed"])
    upd = np.nonzero(kind == 1)[0].astype(np.int32)
    return kind, vals, upd


def cpu_reference_mcf(kind, vals, upd, max_seconds=20.0):
    """Time the compiled reference smoother (all host threads) on a bounded sample."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    c = MCF_CFG
    cores = os.cpu_count() or 1
    nvox = len(upd) * c["bsx"] ** 3
    if oracle.ref_available():
        try:
            oracle.ref()
            kind_s = "reference"
        except OSError:
            kind_s = "port"
    else:
        kind_s = "port"
    if kind_s == "reference":
        oracle.ref().ref_init(cores)
        # warm-up: 2 iterations
        oracle.mcf_reference((c["res"],) * 3, c["bsx"], kind, vals, upd, 2, c["dt"])
        times, it_done = [], 0
        t_start = time.perf_counter()
        while True:
            _, secs = oracle.mcf_reference((c["res"],) * 3, c["bsx"], kind, vals, upd, 4, c["dt"])
            times.append(secs)
            it_done += 4
            if time.perf_counter() - t_start > max_seconds * 0.5 or len(times) >= 5:
                break
        secs = statistics.median(times)
        rate = nvox * 4 / secs / 1e9
        sample = (f"reference applyChannelPdeFast<float> MCF 8-colour on the full 512^3 workload, "
                  f"4 iterations per call, median of {len(times)} calls")
    else:
        t = time.perf_counter()
        oracle.mcf_oracle((c["res"] // c["bsx"],) * 3, c["bsx"], kind, vals, upd, 2, c["dt"])
        secs = time.perf_counter() - t
        rate = nvox * 2 / secs / 1e9
        sample = "C restatement (oracle) of the smoother, full 512^3 workload, 2 iterations"
    return {"value": rate, "unit": "Gvoxel/s/iter", "cores": cores, "kind": kind_s,
            "sample": sample}


def bench_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    kind, vals, upd = mcf_scene()
    cb = cpu_reference_mcf(kind, vals, upd, max_seconds=60.0)
    c = MCF_CFG
    nvox = len(upd) * c["bsx"] ** 3
    # steps: each a full 20-iteration call would take minutes on few cores;
    # the per-iteration rate is the metric, measured over 4-iteration calls.
    line = {"metric": METRIC, "value": cb["value"], "unit": "Gvoxel/s/iter", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": nvox * c["iters"] / (cb["value"] * 1e9) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded sphere-union SDF)", "impl": "reference",
            "config": {"workload": "mcf_512_b16_spheres64_band4_it20", "active_voxels": nvox,
                       "parallelism": "cpu"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "Gvoxel/s/iter", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def bench_mcf(args):
    import torch
    import msbg_gpu
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    c = MCF_CFG
    kind, vals, upd = mcf_scene()
    nb1 = c["res"] // c["bsx"]
    nvox = len(upd) * c["bsx"] ** 3
    ctx = msbg_gpu.Context(local)
    L = msbg_gpu.lib()

    # --- resident-data timing through the device entry point -----------------
    ctx.set_topology(c["res"], c["res"], c["res"], c["bsx"])
    ctx.upload_channel(1, 0, kind, vals, c["band"], -c["band"])
    slot = np.where(kind == 1, np.cumsum(kind == 1) - 1, np.where(kind == 2, -2, np.where(kind == 3, -3, -1))).astype(np.int32)
    bx, by, bz = upd % nb1, (upd // nb1) % nb1, upd // (nb1 * nb1)
    col = (bx & 1) + 2 * (by & 1) + 4 * (bz & 1)
    order = np.argsort(col, kind="stable")
    clist = upd[order]
    cstart = np.zeros(9, np.int32)
    cstart[1:] = np.cumsum(np.bincount(col, minlength=8))
    dev = torch.device("cuda", local)
    pool = torch.from_numpy(vals).to(dev)
    slot_t = torch.from_numpy(slot).to(dev)
    clist_t = torch.from_numpy(clist.astype(np.int32)).to(dev)
    import ctypes as C
    stream = torch.cuda.current_stream()

    def step():
        rc = L.msbg_gpu_pde_mcf_device(ctx._h, C.c_void_p(pool.data_ptr()),
                                       C.c_void_p(slot_t.data_ptr()), C.c_void_p(clist_t.data_ptr()),
                                       cstart.ctypes.data_as(C.POINTER(C.c_int)), nb1, nb1, nb1,
                                       c["bsx"], c["band"], -c["band"], c["iters"], c["dt"], 0,
                                       C.c_void_p(stream.cuda_stream))
        if rc:
            raise RuntimeError(f"mcf rc={rc}")

    launches_per_step = c["iters"] * int((np.diff(cstart) > 0).sum())
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            step()
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    ctx.sync()  # raises if a kernel reported a bounded wait that gave up
    if args.profile:
        ctx.close()
        return
    if dist:
        t = torch.tensor([ms], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        dist.barrier()
    torch.cuda.synchronize()
    clocks = clk.summary()
    ms_step = ms / args.steps
    rate = nvox * c["iters"] / (ms_step * 1e-3) / 1e9 * ws  # whole job
    hbm, _, pk_kind = peaks()
    alg_bytes_step = 8.0 * nvox * c["iters"]
    achieved = alg_bytes_step / (ms_step * 1e-3) / 1e9
    tpc = read_traffic("mcf_colour_kernel_512_b16.txt")
    cells_per_launch = nvox / 8.0
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_kind": pk_kind,
            "traffic": tpc * cells_per_launch if tpc else None,
            "alg_bytes_per_launch": 8.0 * cells_per_launch,
            "kernel": "mcf_colour_kernel<16>"}

    # --- end to end through the C ABI with pinned host buffers ----------------
    host_in = torch.from_numpy(vals).pin_memory()
    host_out = torch.empty_like(host_in).pin_memory()
    kind_c = np.ascontiguousarray(kind)
    upd_c = np.ascontiguousarray(upd)
    pf = C.POINTER(C.c_float)

    def e2e_step():
        rc = L.msbg_gpu_upload_channel(ctx._h, 2, 0, kind_c.ctypes.data_as(C.POINTER(C.c_int8)),
                                       None, C.cast(C.c_void_p(host_in.data_ptr()), pf),
                                       c["band"], -c["band"])
        rc = rc or L.msbg_gpu_pde_mcf(ctx._h, 2, upd_c.ctypes.data_as(C.POINTER(C.c_int)),
                                      len(upd_c), c["iters"], c["dt"], 0)
        rc = rc or L.msbg_gpu_download_channel(ctx._h, 2, None,
                                               C.cast(C.c_void_p(host_out.data_ptr()), pf))
        rc = rc or L.msbg_gpu_sync(ctx._h)
        if rc:
            raise RuntimeError(f"e2e rc={rc}: {L.msbg_gpu_last_error(ctx._h)}")

    for _ in range(max(1, args.warmup)):
        e2e_step()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = (time.perf_counter() - t0) / args.steps
    if dist:
        t = torch.tensor([e2e_s], device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    e2e_rate = nvox * c["iters"] / e2e_s / 1e9 * ws
    h2d = vals.nbytes + kind.nbytes * 4 + upd.nbytes  # values + slot map + block list
    d2h = vals.nbytes

    cb = None
    if rank == 0 and ws == 1 and not args.no_cpu:
        cb = cpu_reference_mcf(kind, vals, upd)
    if rank == 0:
        line = {"metric": METRIC, "value": rate, "unit": "Gvoxel/s/iter", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded sphere-union SDF, 64 spheres)",
                "config": {"workload": "mcf_512_b16_spheres64_band4_it20", "active_voxels": nvox,
                           "value_blocks": int(len(upd)), "iters_per_step": c["iters"],
                           "l2": "inputs larger than L2 (%.0f MB)" % (vals.nbytes / 1e6),
                           "parallelism": f"replicas{ws}"},
                "gpu_launches": launches_per_step * args.steps,
                "roofline": roof, "clocks": clocks,
                "e2e": {"value": e2e_rate, "unit": "Gvoxel/s/iter", "h2d_bytes_per_step": int(h2d),
                        "d2h_bytes_per_step": int(d2h)},
                "cpu_baseline": cb}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mcf", choices=["mcf"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--profile", action="store_true",
                    help="only the resident-data steps (for ncu captures); prints nothing")
    args = ap.parse_args()
    if args.impl == "reference":
        bench_reference(args)
    else:
        bench_mcf(args)


if __name__ == "__main__":
    main()
