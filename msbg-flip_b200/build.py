"""In-tree build of the sm_100a solver library (libmsbg_gpu.so) and of the
synthetic-scene library (libmsbg_scene.so).

Compiles every CUDA/C++ source under csrc/ with nvcc for sm_100a and links
them, with the static CUDA runtime, into ``libmsbg_gpu.so`` next to this file;
compiles scene/scene.cpp (host C++/OpenMP, the seeded input generators) into
``libmsbg_scene.so``.  Run ``python msbg-flip_b200/build.py`` or call
:func:`build`.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OBJ = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libmsbg_gpu.so")
SCENE_SRC = os.path.join(HERE, "scene", "scene.cpp")
SCENE_LIB = os.path.join(HERE, "libmsbg_scene.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-fopenmp,-O3",
          "-I" + os.path.join(ROOT, "include"), "-I" + CSRC]


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(cand):
        raise RuntimeError("nvcc not found")
    return cand


def _sources():
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, f))
    return out


def _headers_mtime() -> float:
    m = 0.0
    for d in (CSRC, os.path.join(ROOT, "include")):
        for f in os.listdir(d):
            if f.endswith((".h", ".cuh", ".hpp")):
                m = max(m, os.path.getmtime(os.path.join(d, f)))
    return m


def build(verbose: bool = False, force: bool = False, extra_flags=None) -> str:
    """Compile all sources (incrementally) and link libmsbg_gpu.so; returns its path."""
    nvcc = _nvcc()
    os.makedirs(OBJ, exist_ok=True)
    hdr = _headers_mtime()
    extra = list(extra_flags or [])
    jobs = []
    objs = []
    for src in _sources():
        obj = os.path.join(OBJ, os.path.basename(src) + ".o")
        objs.append(obj)
        stale = force or not os.path.exists(obj) or \
            os.path.getmtime(obj) < max(os.path.getmtime(src), hdr)
        if stale:
            lang = [] if src.endswith(".cu") else ["-x", "cu"] if False else []
            cmd = [nvcc] + ARCH + COMMON + extra + lang + ["-c", src, "-o", obj]
            jobs.append(cmd)

    def run(cmd):
        if verbose:
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("compile failed:\n" + " ".join(cmd) + "\n" + r.stdout + r.stderr)
        if verbose and (r.stdout or r.stderr):
            print(r.stdout + r.stderr, flush=True)

    with ThreadPoolExecutor(max_workers=max(1, min(8, os.cpu_count() or 1))) as ex:
        list(ex.map(run, jobs))
    # relink when a source was compiled, added or removed
    stamp = os.path.join(OBJ, "objects.txt")
    listed = open(stamp).read() if os.path.exists(stamp) else ""
    if jobs or force or not os.path.exists(LIB) or listed != "\n".join(objs):
        cmd = [nvcc] + ARCH + ["-shared", "-o", LIB] + objs + \
            ["-Xcompiler", "-fopenmp", "-lgomp", "-cudart", "static"]
        run(cmd)
        with open(stamp, "w") as f:
            f.write("\n".join(objs))
    hdr_scene = os.path.getmtime(os.path.join(ROOT, "include", "msbg_scene.h"))
    if force or not os.path.exists(SCENE_LIB) or \
            os.path.getmtime(SCENE_LIB) < max(os.path.getmtime(SCENE_SRC), hdr_scene):
        run(["g++", "-O3", "-std=c++17", "-fPIC", "-fopenmp", "-shared",
             "-I" + os.path.join(ROOT, "include"), SCENE_SRC, "-o", SCENE_LIB])
    return LIB


if __name__ == "__main__":
    p = build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(p)
