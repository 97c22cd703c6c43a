#!/usr/bin/env python
"""Benchmark of the B200 sparse block-grid PDE solver.

Default workload ``mgpcg`` - the FLIP pressure solve on a 2-level adaptive
MSBG at 1024^3 effective resolution: 32^3 base blocks, level 0 within 64
voxels of the liquid surface and 2x coarser elsewhere, liquid = half-space
z < 0.4 plus 32 seeded spheres, 8 seeded solid cuboids, Dirichlet p = 0 in
air, Neumann at walls and solids, RHS = MAC divergence of 16 random Fourier
modes (|k|_inf 1..8, N(0,1) amplitudes).

One step = one MGPCG solve from p = 0 to a TRUE relative residual of 1e-6
(|b - A x| / |b| recomputed in FP64): V(2,2) preconditioner, FP32 level-0
vectors, the solution accumulated in FP64 with reliable residual
replacement, FP64 inner products, FP64 coarsest solve.  value = liquid cells
x PCG iterations / device solve time (Gvoxel/s per iteration); ms_per_step
is the time to 1e-6.  Beside it, in the same line, each over --steps timed
calls after one warm-up:
  - the plain FP32 solve that stops on its recursive residual (the
    reference's criterion; its true residual stalls near 1e-4);
  - FP16 and BF16 level-0 storage under FP64 iterative refinement;
  - the learned variants (networks trained in this run on the GPU);
  - the error against the FP64 oracle, on the same scene family at 256^3
    (a CPU FP64 solve at 1024^3 is out of reach; stated as a proxy);
  - the same solve on the reference's runnable analogue (1024^3 with 16^3
    base blocks: the reference's smoother aborts for 32^3 blocks,
    src/msbg3.cpp:1692-1749), next to the reference's own CPU solver on it;
  - the mean-curvature-flow smoother at 512^3 (16^3 blocks, band +-4 around
    64 seeded spheres, 20 iterations, dt 0.1) with its roofline and the
    reference's CPU smoother on the same input.

  - the particle splatting that produces the smoother's input in the
    reference's demo (1024^3, 16^3 blocks, 4096 instances of a 4096-point
    seeded cloud), next to the reference's own demo code on 1024 instances.

``--workload mcf`` benches only the smoother, ``--workload splat`` only the
splatting, ``--workload g2p_mr`` only G2P on the 3-level grid; ``--workload c3`` / ``c5`` the
2048^3 mixed-precision and 4096^3 three-level configurations (one JSON line
of figures each, see bench_large).
``--impl reference`` times the reference's own CPU implementation (compiled
from its sources into oracle/_ref/libmsbg_ref.so) with all host threads.

Multi-GPU: independent replicas, one per rank (the solve does not shard in
this build); value = all ranks' work / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import ctypes as C
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

PS_CFG = dict(res=1024, bsx0=32, n_levels=2, z_liquid=0.4, n_spheres=32, r_min=0.03, r_max=0.1,
              n_cuboids=8, n_modes=16, k_max=8, band=64.0, seed=2024, tol=1e-6, n_pre=2,
              n_post=2, inner=3)
# the reference's runnable analogue: same scene with 16^3 base blocks (its
# smoother aborts for 32^3 blocks, src/msbg3.cpp:1692-1749)
PS_SAME_CFG = dict(PS_CFG, bsx0=16)
REF_ITERS = 2        # PCG iterations per timed reference call
# the scene family at 256^3 where the FP64 oracle solves in seconds
ERR_RES = 256

MCF_CFG = dict(res=512, bsx=16, n_spheres=64, rmin=20.0, rmax=60.0, band=4.0, dilate=1,
               seed=1234, iters=20, dt=0.1)

# 2048^3: the 1024^3 scene family at twice the resolution (~4e8 active cells),
# level-0 vectors in FP16 and in BF16 under FP64 refinement
C3_CFG = dict(PS_CFG, res=2048)
# 4096^3, 3 levels, fine band of 48 voxels around a wavy free surface
# z = (0.3 + 0.05 sum of 8 seeded sinusoids) * res plus 256 seeded spheres of
# radius 20-60 voxels, no obstacles; FP16 storage with FP64 refinement and
# the learned guess and correction, against plain FP32 on the same GPU.  A
# block is fine when its centre lies within 48 voxels of the surface: the
# scene's band adds half a block diagonal (27.7 voxels for 32^3 blocks) to
# the distance it is given, so it is given 48 - 27.7.
C5_CFG = dict(PS_CFG, res=4096, n_levels=3, band=48.0 - 16 * 3 ** 0.5, z_liquid=0.3,
              n_spheres=256, r_min=20 / 4096, r_max=60 / 4096, n_cuboids=0, wave_amp=0.05,
              n_waves=8, seed=4096)


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


def read_profile_value(name, key):
    """A `key=value` line of a committed ncu summary under profiles/."""
    p = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(p):
        return None
    for line in open(p):
        if line.startswith(key + "="):
            return float(line.split("=")[1])
    return None


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def init_dist(ws, backend="nccl", timeout_s=300):
    """Process group of the replicas (one per GPU; gloo for CPU tests).  A
    rank that fails or never arrives ends the others' next collective with an
    error after timeout_s."""
    if ws <= 1:
        return None
    import datetime

    import torch.distributed as dist
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
    return dist


def max_over_ranks(dist, v, dev):
    if not dist:
        return v
    import torch
    t = torch.tensor([v], device=dev, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload_name(c):
    return f"flip_pressure_mgpcg_{c['res']}_b{c['bsx0']}_{c['n_levels']}lvl"


# ---------------------------------------------------------------------------
# pressure workload
# ---------------------------------------------------------------------------
def ps_scene(cfg):
    import msbg_gpu
    return msbg_gpu.PressureScene(cfg["res"], cfg["bsx0"], cfg["n_levels"], cfg["z_liquid"],
                                  cfg["n_spheres"], cfg["r_min"], cfg["r_max"], cfg["n_cuboids"],
                                  cfg["n_modes"], cfg["k_max"], cfg["band"], cfg["seed"],
                                  cfg.get("wave_amp", 0.0), cfg.get("n_waves", 0))


def ps_stats(ctx):
    import msbg_gpu
    L = msbg_gpu.lib()
    st = msbg_gpu.PressureStats()
    ctx._check(L.msbg_gpu_pressure_stats(ctx._h, C.byref(st)), "stats")
    return st


def solve_params(c, **kw):
    import msbg_gpu
    return msbg_gpu.solve_params(nPre=c["n_pre"], nPost=c["n_post"], tol=c["tol"],
                                 innerIter=c["inner"], useGraph=1, **kw)


def timed_solves(ctx, params, warmup, steps):
    """warmup untimed solves, then `steps` solves; their solve infos."""
    for _ in range(warmup):
        ctx.pressure_solve(params)
    return [ctx.pressure_solve(params) for _ in range(steps)]


def summarize(infos, fluid):
    secs = sum(i.solveSeconds for i in infos)
    its = sum(i.iterations for i in infos)
    return {"ms": secs / len(infos) * 1e3, "gvoxel_s_iter": fluid * its / secs / 1e9,
            "calls": len(infos), "pcg_iterations": [i.iterations for i in infos][:3],
            "refinements": infos[-1].refinements, "status": max(i.status for i in infos),
            "true_rel_residual": max(i.relResidual for i in infos)}


def ref_pressure_rate(cfg, max_seconds=40.0):
    """The reference's solvePressureFLIP (all host threads) on a scene:
    prepare (untimed), one warm-up iteration, then calls of REF_ITERS PCG
    iterations until max_seconds/2 or 3 calls.  Liquid cells are counted
    from the reference's own prepared flags."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    cores = os.cpu_count() or 1
    if not oracle.ref_available():
        return {"value": None, "unit": "Gvoxel/s/iter", "cores": cores, "kind": "reference",
                "sample": "unavailable: oracle/_ref/libmsbg_ref.so not built"}
    import ref_pressure
    oracle.ref().ref_init(cores)
    scene = ps_scene(cfg)
    r = ref_pressure.RefPressure(scene)
    nfl = int(r.liquid().sum())
    r.solve(max_iter=1)  # warm-up (allocations inside the first V-cycle)
    times, iters, rr = [], [], None
    t0 = time.perf_counter()
    while True:
        it, rr, secs = r.solve(max_iter=REF_ITERS)
        times.append(secs)
        iters.append(it)
        if time.perf_counter() - t0 > max_seconds * 0.5 or len(times) >= 3:
            break
    # its two hot routines, one call each after a warm-up call: the level-0
    # operator (multiplyLaplacianMatrixOpt) and the smoother (relax: one
    # red-black block sweep of 5 inner sweeps, src/msbg3.cpp:2245-2369)
    comp = {}
    x0 = (np.random.default_rng(1).uniform(-1, 1, r.packed_size(0)) * r.liquid()).astype(
        np.float32)
    r.set(ref_pressure.CH_FLOAT_3, x0)
    r.set(ref_pressure.CH_FLOAT_2, x0)
    for name, fn in (("matvec", lambda: r.multiply(0, ref_pressure.CH_FLOAT_3,
                                                   ref_pressure.CH_FLOAT_6)),
                     ("relax_sweep", lambda: r.relax(0, ref_pressure.CH_FLOAT_3,
                                                     ref_pressure.CH_FLOAT_2,
                                                     ref_pressure.CH_FLOAT_6, 1))):
        fn()
        t1 = time.perf_counter()
        fn()
        dt1 = time.perf_counter() - t1
        comp[name] = {"ms": dt1 * 1e3, "gvoxel_s": nfl / dt1 / 1e9}
    prep = r.prep_seconds
    r.close()
    return {"value": nfl * sum(iters) / sum(times) / 1e9, "unit": "Gvoxel/s/iter",
            "cores": cores, "kind": "reference", "liquid_cells": nfl, "components": comp,
            "sample": (f"reference solvePressureFLIP (V(2,2)-PCG, src/msbg3.cpp:3098) on "
                       f"{workload_name(cfg)}: {len(times)} calls of {REF_ITERS} PCG "
                       f"iterations after a 1-iteration warm-up; {nfl} liquid cells (its own "
                       f"flags); prepare {prep:.1f} s not counted; |r|/|b| after "
                       f"{REF_ITERS} iterations {rr:.3g} (it does not reach 1e-6)")}


def bench_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return
    if args.workload == "mcf":
        return bench_reference_mcf(args)
    if args.workload == "g2p_mr":
        # the reference's G2P (src/flip_sim.cpp) does not compile here: the CPU
        # restatement of it is timed in its place
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle
        res, bsx, nl, n_part = 512, 16, 3, 1_000_000
        nb = res // bsx
        b = np.arange(nb ** 3)
        r = np.sqrt((b % nb - 12.5) ** 2 + ((b // nb) % nb - 15.5) ** 2 + (b // (nb * nb) - 17.5) ** 2)
        lev = np.where(r < 7, 0, np.where(r < 12, 1, 2)).astype(np.int32)
        _, n = oracle.mr_layout([nb] * 3, bsx, lev)
        rng = np.random.default_rng(21)
        vel = rng.standard_normal(3 * n).astype(np.float32)
        d, k = oracle.mr_dist([nb] * 3, bsx, lev, nl)
        p = np.zeros(n_part, [("pos", "<f4", 3), ("vel", "<f4", 3), ("phase", "<i4")])
        p["pos"] = rng.uniform(0, res, (n_part, 3)).astype(np.float32)
        times = []
        for _ in range(max(args.steps, 1)):
            t0 = time.perf_counter()
            oracle.mr_g2p((res,) * 3, bsx, lev, p, vel, vel, d, k, 0.95)
            times.append(time.perf_counter() - t0)
        v = n_part / float(np.median(times)) / 1e6
        cb = {"value": v, "unit": "Mparticles/s", "cores": 1, "kind": "port",
              "sample": f"{n_part} particles of g2p_multires_512_b16_3lvl, CPU restatement "
                        "(oracle/msbg_oracle_flip_mr.c), one thread, median of "
                        f"{len(times)} calls"}
        print(json.dumps({"metric": "G2P rate on a 3-level grid (interpVec3MSBG blend)",
                          "value": v, "unit": "Mparticles/s", "n_gpus": args.gpus,
                          "steps": args.steps, "warmup": 0, "ms_per_step": n_part / v / 1e3,
                          "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                          "dtype": "f32", "data": "synthetic",
                          "config": {"workload": "g2p_multires_512_b16_3lvl"},
                          "impl": "reference", "cpu_baseline": cb,
                          "e2e": {"value": v, "unit": "Mparticles/s", "h2d_bytes_per_step": 0,
                                  "d2h_bytes_per_step": 0}}), flush=True)
        return
    if args.workload == "splat":
        cb = splat_reference_rate()
        if cb is None:
            print(json.dumps({"impl": "reference", "unavailable":
                              "oracle/_ref/libmsbg_splatref.so was not built"}), flush=True)
            return
        print(json.dumps({
            "metric": "particle splat rate (16-bit render density, the smoother's input)",
            "value": cb["value"], "unit": "Mparticles/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded point cloud, the demo's instance construction)",
            "impl": "reference", "config": {"workload": splat_workload_name(),
                                            "parallelism": "cpu"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "Mparticles/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}), flush=True)
        return
    c = dict(PS_SAME_CFG)
    cb = ref_pressure_rate(c, max_seconds=60.0)
    kind, vals, upd = mcf_scene()
    mcf = cpu_reference_mcf(kind, vals, upd)
    line = {"metric": METRIC, "value": cb["value"], "unit": "Gvoxel/s/iter", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded free-surface pressure problem)", "impl": "reference",
            "config": {"workload": workload_name(c),
                       "note": ("the reference's runnable analogue of "
                                f"{workload_name(PS_CFG)}: same scene with 16^3 base blocks "
                                "(its smoother aborts for 32^3 blocks)"),
                       "time_to_1e-6": "not reached (the reference MGPCG stalls)",
                       "mcf_512_b16": mcf, splat_workload_name(): splat_reference_rate(),
                       "parallelism": "cpu"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "Gvoxel/s/iter", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# training sets, from the refined solver on seeded sphere-union instances at
# 512^3 (64 spheres, radii 20-60 voxels, 32^3 base blocks, 2 levels): the
# guess network's (RHS, solution) pairs on 500 spread-out 16^3 tiles each; the
# correction network's (residual, error) pairs after a V-cycle at PCG
# iterations 0, 1 and 2, 166 tiles each
LEARN_CFG = dict(res=512, seeds=(100, 101, 102, 103), pairs_per_instance=500, epochs=60,
                 batch=64, lr=2e-3)


def learned_variants(ctx, c, scene, fluid, steps, prepare=None):
    """Train the guess and correction networks on the GPU, then time the
    learned solves of the bench problem (FP64 refinement to 1e-6), one
    warm-up and `steps` timed calls each."""
    import torch
    import msbg_gpu
    L = LEARN_CFG
    vc = dict(nPre=c["n_pre"], nPost=c["n_post"], innerIter=c["inner"])
    t0 = time.perf_counter()
    G, K = [], []
    for sd in L["seeds"]:
        ctx.pressure_prepare(msbg_gpu.PressureScene(L["res"], 32, 2, 0.0, 64, 20 / 512, 60 / 512, 8,
                                                    16, 8, 32.0 * L["res"] / 512, sd))
        ctx.pressure_solve(tol=1e-6, maxRefine=4)
        G.append(msbg_gpu.collect_training_pairs(ctx, L["pairs_per_instance"]))
        for k in (0, 1, 2):
            K.append(msbg_gpu.collect_correction_pairs(ctx, L["pairs_per_instance"] // 3, k, **vc))
    cat = lambda P: [torch.cat([q[j] for q in P]) for j in range(3)]
    G, K = cat(G), cat(K)
    data_s = time.perf_counter() - t0
    net, corr = msbg_gpu.Cnn(ctx.device), msbg_gpu.Cnn(ctx.device)
    t0 = time.perf_counter()
    losses = msbg_gpu.train_cnn(net, *G, epochs=L["epochs"], batch=L["batch"], lr=L["lr"], seed=1)
    closs = msbg_gpu.train_cnn(corr, *K, epochs=L["epochs"], batch=L["batch"], lr=L["lr"], seed=2)
    torch.cuda.synchronize()
    train_s = time.perf_counter() - t0
    rel = lambda ls, T, M: (ls[-1] / float((T * T * M).sum() / M.sum())) ** 0.5
    if prepare:
        prepare()
    else:
        ctx.pressure_prepare(scene)
    ctx.pressure_set_cnn(net)
    ctx.pressure_set_correction_cnn(corr)
    out = {"pairs": int(G[0].shape[0]), "correction_pairs": int(K[0].shape[0]),
           "epochs": L["epochs"], "data_seconds": data_s, "train_seconds": train_s,
           "final_rel_loss": rel(losses, G[1], G[2]),
           "correction_final_rel_loss": rel(closs, K[1], K[2]),
           "network": "4 x conv3^3 16ch ReLU, BF16 tcgen05 implicit GEMM, FP32 accumulate"}
    for name, storage, mode in (("f32_vectors_learned_guess", msbg_gpu.F32, 1),
                                ("f16_vectors_learned_guess", msbg_gpu.F16, 1),
                                ("f32_vectors_learned_correction", msbg_gpu.F32, 2),
                                ("f32_vectors_learned_guess_and_correction", msbg_gpu.F32, 3)):
        vp = solve_params(c, storage=storage, maxRefine=30, learned=mode)
        infos = timed_solves(ctx, vp, 1, steps)
        s = summarize(infos, fluid)
        s["fallback_to_plain"] = max(i.learnedFallback for i in infos)
        s["initial_rel_residual"] = infos[-1].initialRelResidual
        out[name] = s
    ctx.pressure_set_cnn(None)
    ctx.pressure_set_correction_cnn(None)
    net.close()
    corr.close()
    return out


def error_vs_oracle(ctx, c):
    """Error of the GPU solutions (FP32, FP16, BF16 level-0 vectors, each to a
    true FP64 residual of 1e-6) against the FP64 oracle (Jacobi-PCG to 1e-11
    on the same system), on the bench's scene family at ERR_RES^3."""
    import msbg_gpu
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    e = dict(c, res=ERR_RES, band=c["band"] * ERR_RES / c["res"])
    scene = ps_scene(e)
    t0 = time.perf_counter()
    xo, _, its, rr = oracle.pressure_oracle(scene, tol=1e-11)
    oracle_s = time.perf_counter() - t0
    ctx.pressure_prepare(scene)
    nrm = float(np.linalg.norm(xo))
    mx = float(np.abs(xo).max())
    out = {"workload": workload_name(e), "oracle": f"FP64 Jacobi-PCG, {its} iterations, "
           f"true |r|/|b| {rr:.2e}, {oracle_s:.1f} s on {os.cpu_count()} host threads"}
    for name, storage in (("f32", msbg_gpu.F32), ("f16", msbg_gpu.F16), ("bf16", msbg_gpu.BF16)):
        info = ctx.pressure_solve(solve_params(c, storage=storage, maxRefine=30))
        x = ctx.pressure_download(fp64=True)
        out[name] = {"rel_l2_err": float(np.linalg.norm(x - xo)) / nrm,
                     "max_abs_err_rel": float(np.abs(x - xo).max()) / mx,
                     "true_rel_residual": info.relResidual, "status": info.status}
    return out


FLIP_CFG = dict(res=256, bsx=16, z_liquid=0.4, ppv=8, air_ppv=1, air_band=8, seed=7, dt=0.02,
                gravity=-9.8, alpha=0.95)


def flip_line(args, ctx):
    """The FLIP transfers either side of the pressure solve on a 256^3
    single-level grid (16^3 blocks): seeded particles (8 liquid per cell below
    z = 0.4 res, 1 air per cell in the 8 cells above), one step of P2G,
    gravity, the pressure-gradient update (with a seeded pressure field) and
    G2P through the C ABI from host arrays, each timed over --steps calls;
    the CPU restatement of the same steps times a sample of the particles."""
    import msbg_gpu
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    c = FLIP_CFG
    res, bsx = c["res"], c["bsx"]
    n = res ** 3
    ctx.set_topology(res, res, res, bsx)
    p = msbg_gpu.flip_particles(res, bsx, c["z_liquid"], c["ppv"], c["air_ppv"], c["air_band"],
                                c["seed"])
    pres = np.random.default_rng(1).standard_normal(n).astype(np.float32)
    steps = max(args.steps, 1)
    out = {"grid": f"{res}^3, {bsx}^3 blocks, single level", "particles": int(len(p))}
    q = p.copy()
    for name, fn in (("p2g", lambda: ctx.flip_p2g(p)),
                     ("gravity", lambda: ctx.flip_gravity(c["gravity"], c["dt"])),
                     ("pressure_gradient", lambda: ctx.flip_pressure_gradient(pres, c["dt"])),
                     ("g2p", lambda: ctx.flip_g2p(q, c["alpha"]))):
        fn()
        t0 = time.perf_counter()
        for _ in range(steps):
            fn()
        dt = (time.perf_counter() - t0) / steps
        per = len(p) if name in ("p2g", "g2p") else n
        out[name] = {"ms": dt * 1e3, ("mparticles_s" if per == len(p) else "mvoxels_s"):
                     per / dt / 1e6}
    out["path"] = "C ABI from host arrays (particle and pressure copies inside each call)"
    # the same on particles resident in device memory (no particle copies)
    import torch
    dpart = torch.from_numpy(p.view(np.uint8).copy()).to(f"cuda:{ctx.device}")
    torch.cuda.synchronize()
    for name, fn in (("p2g", lambda: ctx.flip_p2g_device(dpart.data_ptr(), len(p))),
                     ("g2p", lambda: ctx.flip_g2p_device(dpart.data_ptr(), len(p),
                                                          c["alpha"]))):
        fn()
        t0 = time.perf_counter()
        for _ in range(steps):
            fn()
        dt = (time.perf_counter() - t0) / steps
        out[name + "_device_particles"] = {"ms": dt * 1e3, "mparticles_s": len(p) / dt / 1e6}
    del dpart
    if not args.no_cpu:
        sample = p[:: max(1, len(p) // 2_000_000)]
        t0 = time.perf_counter()
        oracle.flip_p2g(res, bsx, sample)
        t_p2g = time.perf_counter() - t0
        vel, mass, beta, _ = oracle.flip_p2g(res, bsx, p[:1])
        t0 = time.perf_counter()
        oracle.flip_g2p(res, bsx, sample, vel, vel, c["alpha"])
        t_g2p = time.perf_counter() - t0
        out["cpu_port"] = {"kind": "port", "cores": 1,
                           "sample": f"{len(sample)} of the particles, CPU restatement "
                                     "(oracle/msbg_oracle_flip.c), one thread",
                           "p2g_mparticles_s": len(sample) / t_p2g / 1e6,
                           "g2p_mparticles_s": len(sample) / t_g2p / 1e6}
    return out


def flip_mr_line(args, ctx):
    """G2P on a 512^3 grid of 16^3 blocks with 3 levels (level 0 within 7
    blocks of a seeded centre, level 1 within 12, level 2 beyond), seeded MAC
    velocity channels and 16 M seeded particles spread over the grid: the
    interpolation of interpVec3MSBG with its fine/coarse blend, timed over
    --steps calls through the C ABI from host arrays and on particles resident
    in device memory (CUDA events on the context's stream); the CPU
    restatement times a sample of the particles."""
    import msbg_gpu
    import torch
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    res, bsx, nl, n_part, alpha = 512, 16, 3, 16_000_000, 0.95
    nb = res // bsx
    b = np.arange(nb ** 3)
    bx, by, bz = b % nb, (b // nb) % nb, b // (nb * nb)
    r = np.sqrt((bx - 12.5) ** 2 + (by - 15.5) ** 2 + (bz - 17.5) ** 2)
    lev = np.where(r < 7, 0, np.where(r < 12, 1, 2)).astype(np.int32)
    ctx.set_topology(res, res, res, bsx, nl, lev)
    n = msbg_gpu.packed_voxels(bsx, lev)
    rng = np.random.default_rng(21)
    vel = rng.standard_normal(3 * n).astype(np.float32)
    old = rng.standard_normal(3 * n).astype(np.float32)
    ctx.flip_mr_channel(msbg_gpu.FLIP_VEL, vel)
    ctx.flip_mr_channel(msbg_gpu.FLIP_VEL_OLD, old)
    p = np.zeros(n_part, msbg_gpu.FLIP_PARTICLE)
    p["pos"] = rng.uniform(0, res, (n_part, 3)).astype(np.float32)
    p["vel"] = rng.standard_normal((n_part, 3)).astype(np.float32)
    steps = max(args.steps, 1)
    out = {"grid": f"{res}^3, {bsx}^3 blocks, {nl} levels ({np.bincount(lev).tolist()} blocks "
                   "per level)", "particles": n_part, "packed_voxels": n}
    q = p.copy()
    ctx.flip_g2p_mr(q, alpha)  # builds the distance channel once
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.flip_g2p_mr(q, alpha)
    dt = (time.perf_counter() - t0) / steps
    out["g2p_host_particles"] = {"ms": dt * 1e3, "mparticles_s": n_part / dt / 1e6,
                                 "h2d_bytes": 28 * n_part, "d2h_bytes": 28 * n_part}
    dev = torch.from_numpy(p.view(np.uint8).copy()).to(f"cuda:{ctx.device}")
    st = torch.cuda.ExternalStream(ctx.stream(), device=f"cuda:{ctx.device}")
    ctx.flip_g2p_mr_device(dev.data_ptr(), n_part, alpha)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(st)
    for _ in range(steps):
        ctx.flip_g2p_mr_device(dev.data_ptr(), n_part, alpha)
    e1.record(st)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    hbm, _, _ = peaks()
    part_bytes = 28 * n_part + 12 * n_part  # particle read + velocity write
    out["g2p_device_particles"] = {
        "ms": ms, "mparticles_s": n_part / (ms * 1e-3) / 1e6,
        "particle_stream_gbs": part_bytes / (ms * 1e-3) / 1e9,
        "particle_stream_frac": part_bytes / (ms * 1e-3) / 1e9 / hbm,
        "note": "a gather: per particle and component 8 level-0, 8 level-L and 8 distance "
                "reads from the grid channels (L2-resident at this size) besides the "
                "particle's own 28 B read and 12 B write"}
    del dev
    # downsampleVelocity from MG level 0 to 1 on the same grid (no solid or
    # void cells), through the C ABI from host arrays
    lv1 = np.maximum(lev, 1)
    n1 = int(((bsx >> lv1.astype(np.int64)) ** 3).sum())
    flags1 = np.zeros(n1, np.uint16)
    ctx.flip_downsample_velocity(1, flags1, vel)
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.flip_downsample_velocity(1, flags1, vel)
    dt = (time.perf_counter() - t0) / steps
    out["downsample_velocity_mg1"] = {"ms": dt * 1e3, "mvoxels_s": n1 / dt / 1e6,
                                      "h2d_bytes": 12 * n + 2 * n1, "d2h_bytes": 12 * n1,
                                      "path": "C ABI from host arrays (copies inside)"}
    if not args.no_cpu:
        sample = p[:: max(1, n_part // 1_000_000)]
        d, k = oracle.mr_dist([nb] * 3, bsx, lev, nl)
        t0 = time.perf_counter()
        oracle.mr_g2p((res,) * 3, bsx, lev, sample, vel, old, d, k, alpha)
        t = time.perf_counter() - t0
        out["cpu_port"] = {"kind": "port", "cores": 1,
                           "sample": f"{len(sample)} of the particles, CPU restatement "
                                     "(oracle/msbg_oracle_flip_mr.c), one thread",
                           "mparticles_s": len(sample) / t / 1e6}
    return out


# the demo's particle splatting (src/msbg_demo.cpp:339-684): rParticle 2,
# nbDist 2, n_base instances of an n_base-point cloud; the reference's demo is
# timed on the first ref_n_base points of the same cloud (ref_n_base^2
# particles)
SPLAT_CFG = dict(res=1024, bsx=16, n_base=4096, test_case=1, seed=11, ref_n_base=1024)


def splat_workload_name(c=SPLAT_CFG):
    return f"splat_{c['res']}_b{c['bsx']}_demo{c['n_base']}x{c['n_base']}"


def splat_reference_rate(c=SPLAT_CFG):
    """The reference's demo code (msbg_test_sparse, compiled from
    src/msbg_demo.cpp with oracle/ref/splat_harness.cpp observing it) on
    ref_n_base instances of the first ref_n_base points of the cloud, all
    host threads: particles / (block allocation + splat + finalisation)."""
    import msbg_gpu
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    if not oracle.splat_reference_available():
        return None
    base = msbg_gpu.splat_base_cloud(c["n_base"], c["seed"])[: c["ref_n_base"]]
    with tempfile.TemporaryDirectory() as d:
        ply = os.path.join(d, "base.ply")
        oracle.write_ply(ply, base)
        r = oracle.splat_reference_demo(ply, c["test_case"], c["bsx"], (c["res"],) * 3)
    n = len(r["pos"])
    t_splat = r["t_final"] - r["t_marked"]
    return {"value": n / t_splat / 1e6, "unit": "Mparticles/s", "cores": os.cpu_count(),
            "kind": "reference",
            "sample": (f"reference msbg_test_sparse (src/msbg_demo.cpp:228-684) on "
                       f"{c['ref_n_base']} instances of the first {c['ref_n_base']} cloud "
                       f"points ({n} particles, {len(r['blocks'])} value blocks), "
                       f"{c['res']}^3, {c['bsx']}^3 blocks: value = particles / (block "
                       f"allocation + splat + finalisation) = {t_splat:.3f} s; marking and "
                       f"particle construction {r['t_marked']:.3f} s")}


def splat_line(args, ctx):
    """The demo's particle splatting on the GPU: positions resident in device
    memory (value) and through the C ABI from host positions with the
    channel downloaded (e2e), each over --steps calls after one warm-up."""
    import torch
    import msbg_gpu
    c = dict(SPLAT_CFG)
    if args.workload == "splat" and args.res:
        c["res"] = args.res
    if args.workload == "splat" and args.splat_base:
        c["n_base"] = args.splat_base
    res3, bsx = (c["res"],) * 3, c["bsx"]
    pos = msbg_gpu.splat_demo_particles(res3, c["n_base"], c["seed"], c["test_case"])
    ctx.set_topology(*res3, bsx)
    steps = max(args.steps, 1)
    dpos = torch.from_numpy(pos).to(f"cuda:{ctx.device}")
    torch.cuda.synchronize()
    kind = ctx.splat_device(7, dpos.data_ptr(), len(pos))
    nval = int((kind == 1).sum())
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.splat_device(7, dpos.data_ptr(), len(pos))
    dt_dev = (time.perf_counter() - t0) / steps
    del dpos
    # end to end: positions in, the channel out, both in page-locked host memory
    hpos = msbg_gpu.pinned_empty(pos.shape, np.float32)
    hpos[:] = pos
    out = msbg_gpu.pinned_empty((nval * bsx ** 3,), np.uint16)
    ctx.splat(7, hpos)
    t0 = time.perf_counter()
    for _ in range(steps):
        ctx.splat(7, hpos)
        ctx.download_channel_u16(7, out)
    dt_e2e = (time.perf_counter() - t0) / steps
    line = {"workload": splat_workload_name(c), "particles": int(len(pos)),
            "value_blocks": nval, "unit": "Mparticles/s",
            "value": len(pos) / dt_dev / 1e6, "ms_per_call": dt_dev * 1e3,
            "path": "msbg_gpu_splat_particles_device (positions in device memory; marking, "
                    "block kinds, binning, splat and finalisation in each call)",
            "e2e": {"value": len(pos) / dt_e2e / 1e6, "unit": "Mparticles/s",
                    "ms_per_call": dt_e2e * 1e3, "h2d_bytes_per_step": int(pos.nbytes),
                    "d2h_bytes_per_step": int(out.nbytes)}}
    if not args.no_cpu:
        line["cpu_baseline"] = splat_reference_rate(c)
    return line


def bench_splat(args):
    import torch
    import msbg_gpu
    torch.cuda.set_device(0)
    ctx = msbg_gpu.Context(0)
    with Clocks(0) as clk:
        s = splat_line(args, ctx)
    ctx.close()
    cb = s.pop("cpu_baseline", None)
    e2e = s.pop("e2e")
    line = {"metric": "particle splat rate (16-bit render density, the smoother's input)",
            "value": s["value"], "unit": "Mparticles/s", "n_gpus": 1, "steps": args.steps,
            "warmup": 1, "ms_per_step": s["ms_per_call"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded point cloud, the demo's instance construction)",
            "config": s, "clocks": clk.summary(), "e2e": e2e, "cpu_baseline": cb}
    print(json.dumps(line), flush=True)


def bench_g2p_mr(args):
    """--workload g2p_mr: G2P on the 3-level 512^3 grid alone (one JSON line)."""
    import torch
    import msbg_gpu
    torch.cuda.set_device(0)
    ctx = msbg_gpu.Context(0)
    with Clocks(0) as clk:
        s = flip_mr_line(args, ctx)
    ctx.close()
    d, h = s["g2p_device_particles"], s["g2p_host_particles"]
    line = {"metric": "G2P rate on a 3-level grid (interpVec3MSBG blend)",
            "value": d["mparticles_s"], "unit": "Mparticles/s", "n_gpus": 1,
            "steps": args.steps, "warmup": 1, "ms_per_step": d["ms"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded velocity channels, uniformly random particles)",
            "config": dict(s, workload="g2p_multires_512_b16_3lvl"), "clocks": clk.summary(),
            "e2e": {"value": h["mparticles_s"], "unit": "Mparticles/s",
                    "h2d_bytes_per_step": h["h2d_bytes"], "d2h_bytes_per_step": h["d2h_bytes"]},
            "cpu_baseline": s.get("cpu_port")}
    print(json.dumps(line), flush=True)


def bench_mgpcg(args):
    import torch
    import msbg_gpu
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = init_dist(ws)
    dev = torch.device("cuda", local)
    c = dict(PS_CFG)
    if args.res:
        c["res"] = args.res
        c["band"] = PS_CFG["band"] * args.res / PS_CFG["res"]
    ctx = msbg_gpu.Context(local)
    scene = ps_scene(c)
    # the caller's per-cell arrays (flags, lower-face coefficients, rhs) in
    # page-locked host memory: input generation, outside every timed region
    arrays = scene.arrays(pinned=True)

    def prepare_arrays():
        ctx.pressure_prepare_arrays(c["res"], c["bsx0"], c["n_levels"], scene.block_levels,
                                    *arrays)

    prepare_arrays()
    st = ps_stats(ctx)
    fluid = int(st.fluid[0])
    # the step: MGPCG to a true FP64 residual of 1e-6, FP32 level-0 vectors
    params = solve_params(c, storage=msbg_gpu.F32, maxRefine=30)
    for _ in range(args.warmup):
        ctx.pressure_solve(params)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    infos = []
    with Clocks(local) as clk:
        for _ in range(args.steps):
            infos.append(ctx.pressure_solve(params))
        torch.cuda.synchronize()
    clocks = clk.summary()
    solve_s = max_over_ranks(dist, sum(i.solveSeconds for i in infos), dev)
    iters = [i.iterations for i in infos]
    ms_step = solve_s / args.steps * 1e3
    rate = fluid * sum(iters) / solve_s / 1e9 * ws
    launches = sum(i.kernelLaunches for i in infos)
    if args.profile:
        ctx.close()
        return
    # end to end through the C ABI from host buffers: the bulk prepare from the
    # per-cell arrays (copy to the GPU, hierarchy built there), the same
    # solve, download of the pressure; averaged over 3 calls
    n_e2e = 3
    # the caller's pressure array (written in place, as CH_PRESSURE is), in
    # page-locked host memory like the inputs
    out = msbg_gpu.pinned_empty(ctx.pressure_download().shape, np.float32)
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    e2e_iters = 0
    for _ in range(n_e2e):
        prepare_arrays()
        inf = ctx.pressure_solve(params)
        e2e_iters += inf.iterations
        ctx.pressure_download(out=out)
    e2e_s = max_over_ranks(dist, (time.perf_counter() - t0) / n_e2e, dev)
    e2e_rate = fluid * (e2e_iters / n_e2e) / e2e_s / 1e9 * ws
    st2 = ps_stats(ctx)
    # the same through the callbacks (the reference's preparePressureSolveFLIP
    # interface): host sampling and hierarchy build, upload, solve, download
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    ctx.pressure_prepare(scene)
    inf_cb = ctx.pressure_solve(params)
    ctx.pressure_download(out=out)
    e2e_cb_s = max_over_ranks(dist, time.perf_counter() - t0, dev)
    st_cb = ps_stats(ctx)
    extras = {}
    roof = None
    cb = None
    if ws == 1 and not args.quick:
        extras, roof, cb = mgpcg_extras(args, ctx, c, scene, st, fluid, prepare_arrays)
    if rank == 0:
        line = {"metric": METRIC, "value": rate, "unit": "Gvoxel/s/iter", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded free-surface pressure problem)",
                "config": {"workload": workload_name(c),
                           "mode": ("MGPCG to a true FP64 residual of 1e-6: V(2,2), FP32 level-0 "
                                    "vectors, FP64 solution with reliable residual replacement, "
                                    "FP64 dots, FP64 coarsest solve"),
                           "time_to_1e-6_ms": ms_step, "pcg_iterations": iters[:3],
                           "true_rel_residual": max(i.relResidual for i in infos),
                           "status": max(i.status for i in infos),
                           "refinements": infos[-1].refinements,
                           "liquid_cells": fluid, "stored_cells_level0": int(st.cells[0]),
                           "mg_levels": int(st.nMgLevels),
                           "prepare_s": st.prepareSeconds, "build_s": st.buildSeconds,
                           "l2": "inputs larger than L2 (%.1f GB operator+vectors)" %
                                 (st.deviceBytesUsed / 1e9),
                           "parallelism": f"replicas{ws}", **extras},
                "gpu_launches": launches,
                "roofline": roof, "clocks": clocks,
                "e2e": {"value": e2e_rate, "unit": "Gvoxel/s/iter",
                        "h2d_bytes_per_step": int(st2.h2dBytes),
                        "d2h_bytes_per_step": int(out.nbytes),
                        "seconds_per_step": e2e_s, "calls": n_e2e,
                        "path": "msbg_gpu_pressure_prepare_arrays (pinned host arrays; "
                                "hierarchy built on the GPU) + msbg_gpu_pressure_solve + "
                                "msbg_gpu_pressure_download",
                        "prepare_s": st2.prepareSeconds, "build_s": st2.buildSeconds,
                        "callbacks": {"value": fluid * inf_cb.iterations / e2e_cb_s / 1e9 * ws,
                                      "seconds_per_step": e2e_cb_s,
                                      "h2d_bytes_per_step": int(st_cb.h2dBytes),
                                      "host_build_s": st_cb.buildSeconds,
                                      "path": "msbg_gpu_pressure_prepare (host callbacks, "
                                              "host build) + solve + download"}},
                "cpu_baseline": cb}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def mgpcg_extras(args, ctx, c, scene, st, fluid, prepare=None):
    """Sub-figures of the default line (one GPU): roofline of the dominant
    kernel, the other solve variants, the learned variants, the reference's
    analogue, the error against the FP64 oracle and the smoother workload."""
    import msbg_gpu
    hbm, _, pk_kind = peaks()
    K = args.steps
    # dominant kernel: the level-0 tile smoother, one sweep timed on its own
    ms_sw, bytes_sw = ctx.pressure_profile(0, 20, c["inner"])
    ms_vc, bytes_vc = ctx.pressure_profile(2, 5, c["inner"])
    ms_mv, bytes_mv = ctx.pressure_profile(1, 20, c["inner"])
    cells0 = int(st.cells[0])
    dpc = read_profile_value("k_smooth_pipe16_mgpcg_b32.txt", "dram_bytes_per_cell")
    roof = {"bound": "hbm", "achieved": bytes_sw / (ms_sw * 1e-3) / 1e9, "peak": hbm,
            "unit": "GB/s", "frac": bytes_sw / (ms_sw * 1e-3) / 1e9 / hbm, "peak_kind": pk_kind,
            "traffic": dpc * cells0 if dpc else None, "alg_bytes_per_sweep": bytes_sw,
            "kernel": "k_smooth_pipe16 (one level-0 pre-smoothing sweep, one launch per pass)",
            "sweep_ms": ms_sw,
            "matvec_achieved_gbs": bytes_mv / (ms_mv * 1e-3) / 1e9,
            "vcycle_achieved_gbs": bytes_vc / (ms_vc * 1e-3) / 1e9,
            "vcycle_frac": bytes_vc / (ms_vc * 1e-3) / 1e9 / hbm}
    x = {}
    variants = {}
    for name, kw in (("f32_plain_recursive_residual", dict(storage=msbg_gpu.F32, maxRefine=0)),
                     ("f16_vectors_fp64_refined", dict(storage=msbg_gpu.F16, maxRefine=30)),
                     ("bf16_vectors_fp64_refined", dict(storage=msbg_gpu.BF16, maxRefine=30))):
        variants[name] = summarize(timed_solves(ctx, solve_params(c, **kw), 1, K), fluid)
    x["variants"] = variants
    if not args.no_learned:
        x["learned"] = learned_variants(ctx, c, scene, fluid, K, prepare)
    # the reference's runnable analogue (16^3 base blocks), GPU and CPU
    s = dict(PS_SAME_CFG, res=c["res"], band=c["band"])
    ctx.pressure_prepare(ps_scene(s))
    st_s = ps_stats(ctx)
    ms_sw, _ = ctx.pressure_profile(0, 5, c["inner"])
    ms_mv, _ = ctx.pressure_profile(1, 5, c["inner"])
    fl_s = int(st_s.fluid[0])
    same = {"workload": workload_name(s),
            "gpu_components": {
                "matvec": {"ms": ms_mv, "gvoxel_s": fl_s / (ms_mv * 1e-3) / 1e9},
                "smooth_sweep": {"ms": ms_sw, "gvoxel_s": fl_s / (ms_sw * 1e-3) / 1e9,
                                 "note": f"one red-black tile sweep of {c['inner']} inner "
                                         "sweeps (the reference's: 5 inner block sweeps)"}},
            "gpu": summarize(timed_solves(ctx, solve_params(s, maxRefine=30), 1, K),
                             int(st_s.fluid[0])),
            "gpu_plain_recursive_residual": summarize(
                timed_solves(ctx, solve_params(s, maxRefine=0), 1, K), int(st_s.fluid[0]))}
    cb = None
    if not args.no_cpu:
        cb = ref_pressure_rate(s)
        same["reference_cpu"] = cb
    x["same_config"] = same
    x["max_err_vs_fp64_oracle"] = error_vs_oracle(ctx, c)
    x["mcf_512_b16"] = mcf_line(args, ctx)
    x["flip_transfers_256_b16"] = flip_line(args, ctx)
    x["g2p_multires_512_b16_3lvl"] = flip_mr_line(args, ctx)
    x[splat_workload_name()] = splat_line(args, ctx)
    return x, roof, cb


def bench_large(args):
    """The 2048^3 (c3) and 4096^3 (c5) configurations on one GPU: the bulk
    prepare (hierarchy built on the GPU), the smoother's level-0 sweep rate (Gvoxel/s per
    smoother iteration) and the time to a true FP64 residual of 1e-6 of each
    variant, one warm-up and --steps timed calls each."""
    import torch
    import msbg_gpu
    torch.cuda.set_device(0)
    c = dict(C3_CFG if args.workload == "c3" else C5_CFG)
    if args.res:
        c["band"] = c["band"] * args.res / c["res"]
        c["res"] = args.res
    ctx = msbg_gpu.Context(0)
    scene = ps_scene(c)
    t0 = time.perf_counter()
    arrays = scene.arrays()  # the caller's per-cell arrays (input generation)
    arrays_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    ctx.pressure_prepare_arrays(c["res"], c["bsx0"], c["n_levels"], scene.block_levels, *arrays)
    prep_s = time.perf_counter() - t0
    del arrays
    st = ps_stats(ctx)
    fluid = int(st.fluid[0])
    free, total = torch.cuda.mem_get_info(0)
    out = {"workload": workload_name(c) + ("_wavy" if c.get("n_waves") else ""),
           "liquid_cells_level0": fluid,
           "active_cells_all_levels": int(sum(st.fluid[m] for m in range(st.nMgLevels))),
           "stored_cells_level0": int(st.cells[0]), "mg_levels": int(st.nMgLevels),
           "scene_arrays_s": arrays_s,
           "prepare_s": prep_s, "build_s": st.buildSeconds,
           "prepare_path": "msbg_gpu_pressure_prepare_arrays (hierarchy built on the GPU)",
           "device_bytes_used": int(st.deviceBytesUsed), "device_free_after_prepare": int(free)}
    hbm, _, _ = peaks()
    for name, storage in (("f32", msbg_gpu.F32), ("f16", msbg_gpu.F16), ("bf16", msbg_gpu.BF16)):
        ms, by = ctx.pressure_profile(0 | (storage << 4), 5, c["inner"])
        out[f"sweep_{name}"] = {"ms": ms, "gvoxel_s_per_smoother_iteration":
                                int(st.cells[0]) / (ms * 1e-3) / 1e9,
                                "hbm_frac": by / (ms * 1e-3) / 1e9 / hbm}
    variants = [("f32_plain_recursive_residual", dict(storage=msbg_gpu.F32, maxRefine=0)),
                ("f32_vectors_fp64_refined", dict(storage=msbg_gpu.F32, maxRefine=30)),
                ("f16_vectors_fp64_refined", dict(storage=msbg_gpu.F16, maxRefine=30)),
                ("bf16_vectors_fp64_refined", dict(storage=msbg_gpu.BF16, maxRefine=30))]
    for name, kw in variants:
        out[name] = summarize(timed_solves(ctx, solve_params(c, **kw), 1, args.steps), fluid)
    if args.workload == "c5" and not args.no_learned:
        def reprepare():
            a = scene.arrays()
            ctx.pressure_prepare_arrays(c["res"], c["bsx0"], c["n_levels"], scene.block_levels,
                                        *a)

        out["learned"] = learned_variants(ctx, c, scene, fluid, args.steps, reprepare)
    print(json.dumps(out), flush=True)
    ctx.close()


# ---------------------------------------------------------------------------
# mean-curvature-flow workload
# ---------------------------------------------------------------------------
def mcf_scene():
    import msbg_gpu
    c = MCF_CFG
    kind, vals = msbg_gpu.sphere_sdf_scene(c["res"], c["bsx"], c["n_spheres"], c["rmin"], c["rmax"],
                                           c["band"], c["dilate"], c["seed"])
    upd = np.nonzero(kind == 1)[0].astype(np.int32)
    return kind, vals, upd


def cpu_reference_mcf(kind, vals, upd, max_seconds=20.0):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle
    c = MCF_CFG
    cores = os.cpu_count() or 1
    if not oracle.ref_available():
        return {"value": None, "unit": "Gvoxel/s/iter", "cores": cores, "kind": "reference",
                "sample": "unavailable: oracle/_ref/libmsbg_ref.so not built"}
    nvox = len(upd) * c["bsx"] ** 3
    oracle.ref().ref_init(cores)
    oracle.mcf_reference((c["res"],) * 3, c["bsx"], kind, vals, upd, 2, c["dt"])
    times = []
    t_start = time.perf_counter()
    while True:
        _, secs = oracle.mcf_reference((c["res"],) * 3, c["bsx"], kind, vals, upd, 4, c["dt"])
        times.append(secs)
        if time.perf_counter() - t_start > max_seconds * 0.5 or len(times) >= 5:
            break
    secs = statistics.median(times)
    return {"value": nvox * 4 / secs / 1e9, "unit": "Gvoxel/s/iter", "cores": cores,
            "kind": "reference",
            "sample": (f"reference applyChannelPdeFast<float> MCF 8-colour on the full 512^3 "
                       f"workload, 4 iterations per call, median of {len(times)} calls")}


def bench_reference_mcf(args):
    kind, vals, upd = mcf_scene()
    cb = cpu_reference_mcf(kind, vals, upd, max_seconds=60.0)
    c = MCF_CFG
    nvox = len(upd) * c["bsx"] ** 3
    line = {"metric": METRIC, "value": cb["value"], "unit": "Gvoxel/s/iter", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": nvox * c["iters"] / (cb["value"] * 1e9) * 1e3 if cb["value"] else None,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded sphere-union SDF)", "impl": "reference",
            "config": {"workload": "mcf_512_b16_spheres64_band4_it20", "active_voxels": nvox,
                       "parallelism": "cpu"},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": "Gvoxel/s/iter", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def mcf_line(args, ctx, dist=None, dev=None, ws=1, local=0):
    """The MCF smoother at 512^3 on the device (resident pool, --steps calls
    of 20 iterations after --warmup), end to end through the C ABI, and the
    reference's CPU smoother on the same input."""
    import torch
    import msbg_gpu
    c = MCF_CFG
    kind, vals, upd = mcf_scene()
    nb1 = c["res"] // c["bsx"]
    nvox = len(upd) * c["bsx"] ** 3
    L = msbg_gpu.lib()
    dev = dev or torch.device("cuda", local)
    slot = np.where(kind == 1, np.cumsum(kind == 1) - 1,
                    np.where(kind == 2, -2, np.where(kind == 3, -3, -1))).astype(np.int32)
    bx, by, bz = upd % nb1, (upd // nb1) % nb1, upd // (nb1 * nb1)
    col = (bx & 1) + 2 * (by & 1) + 4 * (bz & 1)
    clist = upd[np.argsort(col, kind="stable")]
    cstart = np.zeros(9, np.int32)
    cstart[1:] = np.cumsum(np.bincount(col, minlength=8))
    pool = torch.from_numpy(vals).to(dev)
    slot_t = torch.from_numpy(slot).to(dev)
    clist_t = torch.from_numpy(clist.astype(np.int32)).to(dev)
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
    # resident channel of the context path, which keeps the face cache of the
    # x halos (msbg_gpu_pde_mcf); the caller-pool entry point above is timed
    # beside it
    ctx.set_topology(c["res"], c["res"], c["res"], c["bsx"])
    ctx.upload_channel(7, 0, kind, vals, c["band"], -c["band"])
    cstream = torch.cuda.ExternalStream(ctx.stream(), device=dev)

    def ctx_step():
        ctx.apply_channel_pde_mcf(7, upd, c["iters"], c["dt"], sync=False)

    for _ in range(max(args.warmup, 3)):
        step()
        ctx_step()
    torch.cuda.synchronize()
    ctx.sync()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with Clocks(local) as clk:
        ev0.record(cstream)
        for _ in range(args.steps):
            ctx_step()
        ev1.record(cstream)
        ctx.sync()
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    ev2, ev3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev2.record(stream)
    for _ in range(args.steps):
        step()
    ev3.record(stream)
    torch.cuda.synchronize()
    ms_device_entry = ev2.elapsed_time(ev3)
    ctx.sync()
    ms = max_over_ranks(dist, ms, dev)
    clocks = clk.summary()
    ms_step = ms / args.steps
    rate = nvox * c["iters"] / (ms_step * 1e-3) / 1e9 * ws
    hbm, _, pk_kind = peaks()
    alg = 8.0 * nvox * c["iters"]
    achieved = alg / (ms_step * 1e-3) / 1e9
    dpc = read_profile_value("mcf_colour_kernel_tma_512_b16.txt", "dram_bytes_per_cell")
    roof = {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "peak_kind": pk_kind,
            "traffic": dpc * nvox / 8.0 if dpc else None,
            "alg_bytes_per_launch": 8.0 * nvox / 8.0,
            "kernel": "mcf_colour_kernel_tma (16^3 FP32 blocks, tensor-box staging)"}
    ctx.set_topology(c["res"], c["res"], c["res"], c["bsx"])  # the C-ABI path needs the raster
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
            raise RuntimeError(f"e2e rc={rc}")

    e2e_step()
    if dist:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = max_over_ranks(dist, (time.perf_counter() - t0) / args.steps, dev)
    cb = None
    if not args.no_cpu and ws == 1:
        cb = cpu_reference_mcf(kind, vals, upd)
    return {"workload": "mcf_512_b16_spheres64_band4_it20", "value": rate,
            "unit": "Gvoxel/s/iter", "ms_per_step": ms_step, "active_voxels": nvox,
            "caller_pool_entry_gvoxel_s_iter":
                nvox * c["iters"] / (ms_device_entry / args.steps * 1e-3) / 1e9,
            "value_blocks": int(len(upd)), "iters_per_step": c["iters"],
            "gpu_launches": launches_per_step * args.steps, "roofline": roof, "clocks": clocks,
            "e2e": {"value": nvox * c["iters"] / e2e_s / 1e9 * ws, "unit": "Gvoxel/s/iter",
                    "h2d_bytes_per_step": int(vals.nbytes + kind.nbytes * 4 + upd.nbytes),
                    "d2h_bytes_per_step": int(vals.nbytes)},
            "cpu_baseline": cb}


def bench_mcf(args):
    import torch
    import msbg_gpu
    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = init_dist(ws)
    dev = torch.device("cuda", local)
    ctx = msbg_gpu.Context(local)
    m = mcf_line(args, ctx, dist, dev, ws, local)
    if rank == 0 and not args.profile:
        line = {"metric": METRIC, "value": m["value"], "unit": "Gvoxel/s/iter", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": m["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic (seeded sphere-union SDF, 64 spheres)",
                "config": {"workload": m["workload"], "active_voxels": m["active_voxels"],
                           "value_blocks": m["value_blocks"], "iters_per_step": m["iters_per_step"],
                           "l2": "inputs larger than L2", "parallelism": f"replicas{ws}"},
                "gpu_launches": m["gpu_launches"], "roofline": m["roofline"],
                "clocks": m["clocks"], "e2e": m["e2e"], "cpu_baseline": m["cpu_baseline"]}
        print(json.dumps(line), flush=True)
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


# ---------------------------------------------------------------------------
# part timings for profiles
# ---------------------------------------------------------------------------
def bench_part(args):
    """One solver part (a level-0 smoothing sweep, the level-0 matvec or a
    V-cycle) of the pressure workload, timed through msbg_gpu_pressure_profile:
    one warm-up call, then --steps calls.  Prints the level-0 cell count so a
    capture's DRAM bytes can be put per cell."""
    import torch
    import msbg_gpu
    torch.cuda.set_device(0)
    c = dict(PS_CFG)
    if args.res:
        c["res"] = args.res
        c["band"] = PS_CFG["band"] * args.res / PS_CFG["res"]
    ctx = msbg_gpu.Context(0)
    ctx.pressure_prepare(ps_scene(c))
    st = ps_stats(ctx)
    what = {"smooth": 0, "matvec": 1, "vcycle": 2}[args.part]
    storage = {"f32": msbg_gpu.F32, "f16": msbg_gpu.F16, "bf16": msbg_gpu.BF16}[args.storage]
    ms, by = ctx.pressure_profile(what | (storage << 4), max(1, args.steps), c["inner"])
    print(json.dumps({"part": args.part, "storage": args.storage, "res": c["res"],
                      "cells_level0": int(st.cells[0]), "ms_per_call": ms,
                      "alg_bytes_per_call": by, "achieved_gbs": by / (ms * 1e-3) / 1e9}),
          flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mgpcg",
                    choices=["mgpcg", "mcf", "splat", "c3", "c5", "g2p_mr"])
    ap.add_argument("--res", type=int, default=0, help="override the pressure resolution")
    ap.add_argument("--splat-base", type=int, default=0,
                    help="points of the splat workload's cloud (n^2 particles)")
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline legs")
    ap.add_argument("--no-learned", action="store_true", help="skip training and timing the learned guess")
    ap.add_argument("--quick", action="store_true",
                    help="only the headline solve and its end-to-end figure")
    ap.add_argument("--profile", action="store_true",
                    help="only the resident-data steps (for ncu captures); prints nothing")
    ap.add_argument("--part", default="", choices=["", "smooth", "matvec", "vcycle"],
                    help="time one solver part of the pressure workload (ncu captures); "
                         "--steps calls after one warm-up call")
    ap.add_argument("--storage", default="f32", choices=["f32", "f16", "bf16"],
                    help="level-0 vector storage of --part")
    args = ap.parse_args()
    if args.part:
        bench_part(args)
    elif args.impl == "reference":
        bench_reference(args)
    elif args.workload == "mcf":
        bench_mcf(args)
    elif args.workload == "splat":
        bench_splat(args)
    elif args.workload == "g2p_mr":
        bench_g2p_mr(args)
    elif args.workload in ("c3", "c5"):
        bench_large(args)
    else:
        bench_mgpcg(args)


if __name__ == "__main__":
    main()
