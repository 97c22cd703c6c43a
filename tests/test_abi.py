"""CPU tests of the C-ABI library: it loads and exports what the headers declare."""
import glob
import os
import re
import subprocess

import numpy as np
import pytest

import msbg_gpu
from conftest import ROOT


def declared_symbols():
    syms = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        for m in re.finditer(r"^\s*(?:const\s+)?[\w\s\*]+?\b(msbg_\w+)\s*\(", src, re.M):
            syms.add(m.group(1))
    return syms


def test_library_exports_every_declared_symbol():
    msbg_gpu.lib()
    out = subprocess.run(["nm", "-D", "--defined-only", msbg_gpu.LIB_PATH], capture_output=True,
                         text=True, check=True).stdout
    exported = {l.split()[-1] for l in out.splitlines() if l.strip()}
    decl = declared_symbols()
    assert len(decl) >= 10
    missing = decl - exported
    assert not missing, missing


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
