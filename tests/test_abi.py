"""CPU tests of the C-ABI library: it loads and exports what the headers declare."""
import glob
import os
import re
import subprocess

import numpy as np
import pytest

import msbg_gpu
from conftest import ROOT


def declared_symbols(header):
    syms = set()
    src = open(os.path.join(ROOT, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(msbg_\w+)\s*\(", src, re.M):
        syms.add(m.group(1))
    return syms


def exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True,
                         check=True).stdout
    return {l.split()[-1] for l in out.splitlines() if l.strip()}


# each header and the library that implements it
LIBS = {"msbg_gpu.h": msbg_gpu.LIB_PATH, "msbg_cnn.h": msbg_gpu.LIB_PATH,
        "msbg_scene.h": msbg_gpu.SCENE_LIB_PATH}


def test_every_header_has_its_library():
    heads = {os.path.basename(h) for h in glob.glob(os.path.join(ROOT, "include", "*.h"))}
    assert heads == set(LIBS)


@pytest.mark.parametrize("header", sorted(LIBS))
def test_library_exports_every_declared_symbol(header):
    msbg_gpu.lib()
    msbg_gpu.scene_lib()
    decl = declared_symbols(header)
    assert len(decl) >= 5
    missing = decl - exported(LIBS[header])
    assert not missing, missing


def test_solver_library_holds_no_scene_generator():
    assert not any(s.startswith("msbg_scene") for s in exported(msbg_gpu.LIB_PATH))


def test_library_is_sm100a():
    out = subprocess.run(["cuobjdump", "--list-elf", msbg_gpu.LIB_PATH], capture_output=True,
                         text=True)
    if out.returncode != 0:
        pytest.skip("cuobjdump unavailable")
    assert "sm_100a" in out.stdout


def test_scene_generator_is_deterministic():
    k1, v1 = msbg_gpu.sphere_sdf_scene(64, 16, n_spheres=4, rmin=5, rmax=12, seed=5)
    k2, v2 = msbg_gpu.sphere_sdf_scene(64, 16, n_spheres=4, rmin=5, rmax=12, seed=5)
    np.testing.assert_array_equal(k1, k2)
    np.testing.assert_array_equal(v1, v2)
    k3, _ = msbg_gpu.sphere_sdf_scene(64, 16, n_spheres=4, rmin=5, rmax=12, seed=6,
                                      with_values=False)
    assert (k1 != k3).any()
    assert set(np.unique(k1)) <= {1, 2, 3}


def test_scene_rejects_bad_arguments():
    with pytest.raises(msbg_gpu.MsbgError):
        msbg_gpu.sphere_sdf_scene(60, 16)
