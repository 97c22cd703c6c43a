"""Generate the golden fixtures of the particle splatting from the reference.

Runs the reference's own particle-splatting demo, msbg_test_sparse
(src/msbg_demo.cpp:228-767), compiled from its source file by
``make -C oracle splat`` (oracle/ref/splat_harness.cpp observes it; it changes
nothing it computes), on seeded base point clouds written as PLY files, and
stores per case:
  pos     the particles the demo splatted (its instance construction of the
          base cloud, src/msbg_demo.cpp:339-385), float32 [n, 3]
  blocks  the value blocks after marking and refinement (ascending bid)
  raw     their voxels after the splat loop: quantised squared distances
  final   their voxels after the distance finalisation (render density)
plus the demo's domain test evaluated by the reference on probe points at
the bounds (``splat_domain.npz``).  Re-run with
``python tests/golden/make_splat_golden.py`` (needs the reference tree to
build the library; the fixtures themselves travel without it).
"""
from __future__ import annotations

import os
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402

# (name, base points, demo test case, bsx, grid)
CASES = [
    ("splat_demo_b8", 48, 1, 8, (64, 64, 64)),
    ("splat_demo_b16", 40, 2, 16, (64, 64, 64)),
    ("splat_demo_b32", 24, 1, 32, (64, 64, 64)),
]


def base_cloud(rng, n):
    """A seeded stand-in for the demo's PLY model: points near an ellipsoid
    surface with a little noise."""
    v = rng.normal(size=(n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return v * np.array([1.0, 0.7, 0.5]) + 0.05 * rng.normal(size=(n, 3))


def domain_probes(res3):
    """Points one and two float steps either side of the demo's domain
    bounds on each axis, plus non-finite and corner points."""
    lo, hi = oracle.splat_domain(res3)
    pts = []
    for k in range(3):
        for b in (lo[k], hi[k]):
            for d in (-2, -1, 0, 1, 2):
                x = np.float32(b)
                for _ in range(abs(d)):
                    x = np.nextafter(x, np.float32(1e9 if d > 0 else -1e9), dtype=np.float32)
                p = np.full(3, 5.0, np.float32)
                p[k] = x
                pts.append(p)
    pts += [np.array(v, np.float32) for v in
            ([np.nan, 5, 5], [5, np.inf, 5], [5, 5, -np.inf], [0, 0, 0], [res3[0], 5, 5])]
    return np.array(pts, np.float32)


def main():
    oracle.build_ref()
    rng = np.random.default_rng(20240611)
    with tempfile.TemporaryDirectory() as d:
        for name, nbase, tc, bsx, res3 in CASES:
            ply = os.path.join(d, name + ".ply")
            oracle.write_ply(ply, base_cloud(rng, nbase))
            r = oracle.splat_reference_demo(ply, tc, bsx, res3)
            assert np.array_equal(r["blocks"], r["active"])
            np.savez_compressed(os.path.join(HERE, name + ".npz"), pos=r["pos"],
                                blocks=r["blocks"], raw=r["raw"], final=r["final"], bsx=bsx,
                                res=np.array(res3), test_case=tc)
            print(name, len(r["pos"]), "particles,", len(r["blocks"]), "blocks")
    res3 = (64, 64, 128)
    pts = domain_probes(res3)
    keep = oracle.splat_reference_in_domain(res3, 16, pts)
    np.savez_compressed(os.path.join(HERE, "splat_domain.npz"), pts=pts, keep=keep,
                        res=np.array(res3))


if __name__ == "__main__":
    main()
