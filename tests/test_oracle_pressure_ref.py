"""The FP64 pressure oracle pinned to the compiled reference (CPU only).

The reference's multiplyLaplacianMatrixOpt (src/msbg3.cpp:1757-1912, cell
kernel 1282-1321) applied to a random vector is compared with the oracle's
independent CSR operator (oracle/msbg_oracle_pressure.c) on the same inputs:
  - a grid with every block at level 0, both sampling the same scene
    callbacks;
  - an adaptive 2-level grid, the oracle reading the reference's own prepared
    level-0 channels (flags, face weights), because the reference samples its
    coarse blocks at unscaled coordinates (src/msbg3.cpp:2494-2503).  Cells on
    a face between blocks of different levels are the documented exception
    (the reference's diagonal there ignores the mixed-level faces,
    src/msbg3.cpp:2686-2731); everywhere else the two agree to FP32 rounding.
"""
import numpy as np
import pytest

import oracle
from refgrid import ADAPTIVE, SINGLE, interface_mask, rel_max

pytestmark = pytest.mark.skipif(not oracle.ref_available(), reason="reference not built")


def _ref_and_x(cfg, seed=1):
    import msbg_gpu
    import ref_pressure as rp

    res, bsx0, nl, band = cfg
    scene = msbg_gpu.PressureScene(res, bsx0, nl, band=band, seed=5)
    R = rp.RefPressure(scene)
    liquid = R.liquid()
    rng = np.random.default_rng(seed)
    x = (rng.uniform(-1, 1, R.packed_size(0)) * liquid).astype(np.float32)
    R.set(rp.CH_FLOAT_3, x)
    R.multiply(0, rp.CH_FLOAT_3, rp.CH_FLOAT_6)
    return scene, R, x, R.get(rp.CH_FLOAT_6)


def test_oracle_operator_equals_reference_on_level0_grid():
    scene, R, x, y_ref = _ref_and_x(SINGLE)
    assert (scene.block_levels == 0).all()
    y = oracle.pressure_apply_oracle(scene, x.astype(np.float64))
    assert rel_max(y, y_ref) <= 1e-6


def test_oracle_operator_equals_reference_away_from_level_interfaces():
    scene, R, x, y_ref = _ref_and_x(ADAPTIVE)
    assert set(np.unique(scene.block_levels)) == {0, 1}
    A = R.array_scene()
    y = oracle.pressure_apply_oracle(A, x.astype(np.float64))
    iface = interface_mask(scene.block_levels, scene.res, scene.bsx0)
    assert rel_max(y, y_ref, ~iface) <= 1e-6
    # the exception is confined to the interface cells
    bad = np.abs(y - y_ref) > 1e-4 * np.abs(y_ref).max()
    assert not (bad & ~iface).any()


def test_oracle_residual_equals_reference():
    import ref_pressure as rp

    scene, R, x, _ = _ref_and_x(SINGLE, seed=2)
    rng = np.random.default_rng(3)
    b = (rng.uniform(-1, 1, len(x)) * R.liquid()).astype(np.float32)
    R.set(rp.CH_FLOAT_2, b)
    R.multiply(0, rp.CH_FLOAT_3, rp.CH_FLOAT_6, ch_b=rp.CH_FLOAT_2)
    r_ref = R.get(rp.CH_FLOAT_6)
    r = b - oracle.pressure_apply_oracle(scene, x.astype(np.float64))
    assert rel_max(r, r_ref, R.liquid()) <= 1e-6


def test_domain_faces_follow_the_reference_operator():
    """The reference's FLIP operator ignores setDomainBoundarySpec_: its
    diagonal (computeDiagonalFLIP_, src/msbg3.cpp:2714-2722) takes the
    callback's coefficient on the lower domain faces and reads the upper ones
    past the grid as 0, whatever the spec.  With a face callback that is 0.5
    everywhere, the oracle without a spec (the rule msbg_topo_desc.domainBc =
    NULL selects) equals the reference's A x for every spec the reference is
    given, including flip_sim's open top (src/flip_sim.cpp:1621)."""
    import ref_pressure as rp
    from refgrid import OpenPool

    s = OpenPool(res=32, bsx0=16, z_liquid=20)
    rng = np.random.default_rng(4)
    for bc in ((rp.DBC_SOLID,) * 6, (rp.DBC_OPEN,) * 6, (1, 1, 1, 0, 1, 1)):
        R = rp.RefPressure(s, dom_bc=bc)
        try:
            x = (rng.uniform(-1, 1, R.packed_size(0)) * R.liquid()).astype(np.float32)
            R.set(rp.CH_FLOAT_3, x)
            R.multiply(0, rp.CH_FLOAT_3, rp.CH_FLOAT_6)
            y_ref = R.get(rp.CH_FLOAT_6)
        finally:
            R.close()
        y = oracle.pressure_apply_oracle(s, x.astype(np.float64))
        assert rel_max(y, y_ref) <= 1e-6, bc
        # the lower faces do count: without them the two differ
        y_solid = oracle.pressure_apply_oracle(s, x.astype(np.float64), domain_bc=[1] * 6)
        assert rel_max(y_solid, y_ref) > 1e-2
