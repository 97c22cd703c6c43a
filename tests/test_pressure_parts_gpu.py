"""Per-call parity of the pressure solver's kernels with the compiled reference.

Each test runs one component entry point of the C ABI (msbg_gpu_matvec,
msbg_gpu_residual, msbg_gpu_restrict, msbg_gpu_prolongate, msbg_gpu_relax,
msbg_gpu_pressure_diagonal) once and compares it with the reference routine it
replaces, called through the reference's own API (oracle/ref/ref_harness.cpp)
on the same inputs:
  - on the grid with every block at level 0 the GPU problem is prepared from
    the reference's own prepared channels (msbg_gpu_pressure_prepare_arrays),
    so both operate on identical flags and face weights, and the callback
    prepare is checked to give the same operator;
  - on the adaptive grid both sample the same scene callbacks.  The
    reference samples its level-1 blocks at unscaled coordinates
    (src/msbg3.cpp:2494-2503), which leaves its coarse-block data
    inconsistent (on this grid it even encloses liquid without air, a
    singular system the GPU prepare rejects), so there the comparison
    covers the cells of level-0 blocks;
  - vectors are 0 off liquid, as both solvers keep them;
  - tolerance: FP32, max |gpu - ref| <= 1e-6 max |ref| per call, everywhere
    the two discretisations coincide.  Cells on a face between blocks of
    different levels are the documented exception (mixed-level ghosts).
"""
import numpy as np
import pytest

import oracle
from refgrid import (ADAPTIVE, SINGLE, block_parity, blocks_without_interface, cell_levels,
                     interface_mask, rel_max)

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not oracle.ref_available(), reason="reference not built")]


class Case:
    def __init__(self, cfg, arrays):
        import msbg_gpu
        import ref_pressure as rp

        res, bsx0, nl, band = cfg
        self.res, self.bsx0 = res, bsx0
        self.scene = msbg_gpu.PressureScene(res, bsx0, nl, band=band, seed=5)
        self.R = rp.RefPressure(self.scene)
        self.ctx = msbg_gpu.Context(0)
        if arrays:
            flags, face, rhs = self.R.level0_arrays()
            self.ctx.pressure_prepare_arrays(res, bsx0, nl, self.scene.block_levels, flags, face,
                                             rhs)
        else:
            self.ctx.pressure_prepare(self.scene)
        bl = self.scene.block_levels
        self.iface = interface_mask(bl, res, bsx0)
        self.h = (2.0 ** cell_levels(bl, bsx0)).astype(np.float32)
        self.n = self.R.packed_size(0)
        assert self.ctx.level_size(0) == self.n
        # cells where both sides hold the same data: every cell with array
        # inputs, the cells of level-0 blocks with callbacks
        self.same = np.ones(self.n, bool) if arrays else cell_levels(bl, bsx0) == 0
        # liquid for both solvers (vectors are 0 elsewhere)
        self.liquid = self.R.liquid() & (self.ctx.diagonal(0) > 0)

    def rand(self, seed, level_mg=0, mask=True):
        rng = np.random.default_rng(seed)
        n = self.R.packed_size(level_mg)
        v = rng.uniform(-1, 1, n).astype(np.float32)
        if mask and level_mg == 0:
            v *= self.liquid
        return v

    def close(self):
        self.ctx.close()
        self.R.close()


@pytest.fixture(scope="module")
def single():
    c = Case(SINGLE, arrays=True)
    yield c
    c.close()


@pytest.fixture(scope="module")
def adaptive():
    c = Case(ADAPTIVE, arrays=False)
    yield c
    c.close()


def test_liquid_cells_and_diagonal_match_reference(single, adaptive):
    import ref_pressure as rp

    for c in (single, adaptive):
        a = c.ctx.diagonal(0)
        assert ((a > 0) == c.R.liquid())[c.same].all()
        D = c.R.get(rp.CH_DIAGONAL)  # 1 / sum of the 6 face weights
        m = c.liquid & ~c.iface & c.same
        assert rel_max(c.h[m] / a[m], D[m]) <= 1e-6


def test_callback_prepare_gives_the_reference_operator():
    import ref_pressure as rp

    c = Case(SINGLE, arrays=False)
    try:
        x = c.rand(11)
        c.R.set(rp.CH_FLOAT_3, x)
        c.R.multiply(0, rp.CH_FLOAT_3, rp.CH_FLOAT_6)
        assert rel_max(c.ctx.matvec(0, x), c.R.get(rp.CH_FLOAT_6)) <= 1e-6
    finally:
        c.close()


@pytest.mark.parametrize("which", ["single", "adaptive"])
def test_matvec_matches_reference(which, single, adaptive):
    import ref_pressure as rp

    c = single if which == "single" else adaptive
    x = c.rand(1)
    c.R.set(rp.CH_FLOAT_3, x)
    c.R.multiply(0, rp.CH_FLOAT_3, rp.CH_FLOAT_6)
    y_ref = c.R.get(rp.CH_FLOAT_6)
    y = c.ctx.matvec(0, x)
    assert rel_max(y, y_ref, ~c.iface & c.same) <= 1e-6
    if which == "single":
        assert not c.iface.any()


@pytest.mark.parametrize("which", ["single", "adaptive"])
def test_residual_matches_reference(which, single, adaptive):
    import ref_pressure as rp

    c = single if which == "single" else adaptive
    x, b = c.rand(2), c.rand(3)
    c.R.set(rp.CH_FLOAT_3, x)
    c.R.set(rp.CH_FLOAT_2, b)
    c.R.multiply(0, rp.CH_FLOAT_3, rp.CH_FLOAT_6, ch_b=rp.CH_FLOAT_2)
    r_ref = c.R.get(rp.CH_FLOAT_6)
    r = c.ctx.residual(0, x, b)
    m = c.liquid & ~c.iface & c.same
    assert rel_max(r, r_ref, m) <= 1e-6
    assert (r[c.ctx.diagonal(0) <= 0] == 0).all()


@pytest.mark.parametrize("which", ["single", "adaptive"])
def test_restriction_matches_reference(which, single, adaptive):
    """Coarsened blocks: the sum over liquid children = 8 x the reference's
    average (OPT_SIMPLE_AVERAGE, src/msbg4.cpp:1562-1566) of a vector that is
    0 off liquid; blocks not coarsened at this step: the same values."""
    import ref_pressure as rp

    c = single if which == "single" else adaptive
    f = c.rand(4)
    n1 = c.R.packed_size(1)
    c.R.set(rp.CH_FLOAT_6, f)
    c.R.set(rp.CH_FLOAT_2, np.zeros(n1, np.float32), 1)
    c.R.downsample(1, rp.CH_FLOAT_6, rp.CH_FLOAT_2)
    avg = c.R.get(rp.CH_FLOAT_2, 1)
    got = c.ctx.restrict(1, f)
    bl = c.scene.block_levels
    coarsened = np.repeat(bl == 0, [(c.bsx0 >> max(int(l), 1)) ** 3 for l in bl])
    expect = np.where(coarsened, 8.0 * avg, avg).astype(np.float32)
    # blocks not coarsened at this step copy their fine values, which for the
    # adaptive grid are the level-1 cells whose data differ (see above)
    cmp = coarsened if which == "adaptive" else None
    assert rel_max(got, expect, cmp) <= 1e-6


@pytest.mark.parametrize("which", ["single", "adaptive"])
def test_prolongation_matches_reference(which, single, adaptive):
    import ref_pressure as rp

    c = single if which == "single" else adaptive
    fine = c.rand(5)
    coarse = c.rand(6, level_mg=1, mask=False)
    c.R.set(rp.CH_FLOAT_3, coarse, 1)
    c.R.set(rp.CH_FLOAT_3, fine, 0)
    c.R.prolongate(0, rp.CH_FLOAT_3, rp.CH_FLOAT_3)
    ref = c.R.get(rp.CH_FLOAT_3, 0)
    got = c.ctx.prolongate(0, coarse, fine, 1.0)
    # coarse cells of blocks without liquid are not held on the GPU; their
    # children are not liquid, so the comparison covers every cell that both
    # sides hold the same data for
    assert rel_max(got, ref, c.same) <= 1e-6


@pytest.mark.parametrize("n_iter,reverse", [(1, 0), (1, 1), (2, 0), (2, 1)])
def test_reference_block_smoother_matches_reference(single, n_iter, reverse):
    """msbg_gpu_relax mode 1 against the reference's relax: blocks red-black,
    5 damped block-local sweeps each, directions alternating, last sweep
    Jacobi (src/msbg3.cpp:1109-1506, 2171-2369)."""
    import ref_pressure as rp

    c = single
    x, b = c.rand(7), c.rand(8)
    c.R.set(rp.CH_FLOAT_3, x)
    c.R.set(rp.CH_FLOAT_2, b)
    c.R.relax(0, rp.CH_FLOAT_3, rp.CH_FLOAT_2, rp.CH_FLOAT_6, n_iter, reverse)
    ref = c.R.get(rp.CH_FLOAT_3)
    got = c.ctx.relax(0, x, b, n_iter, reverse, inner=5, mode=1, omega=c.R.omega())
    assert rel_max(got, ref) <= 1e-6


def test_reference_block_smoother_on_adaptive_grid(adaptive):
    """One relax call on the 2-level grid: the level-0 blocks of the first
    parity pass that touch no level interface match (the second pass reads
    halos the interface blocks have already changed)."""
    import ref_pressure as rp

    c = adaptive
    x, b = c.rand(9), c.rand(10)
    c.R.set(rp.CH_FLOAT_3, x)
    c.R.set(rp.CH_FLOAT_2, b)
    c.R.relax(0, rp.CH_FLOAT_3, rp.CH_FLOAT_2, rp.CH_FLOAT_6, 1, 0)
    ref = c.R.get(rp.CH_FLOAT_3)
    got = c.ctx.relax(0, x, b, 1, 0, inner=5, mode=1, omega=c.R.omega())
    bl = c.scene.block_levels
    first = ((block_parity(c.res, c.bsx0) == 1) & blocks_without_interface(bl, c.res, c.bsx0)
             & (bl == 0))
    assert first.any()
    cells = np.repeat(first, [(c.bsx0 >> int(l)) ** 3 for l in bl])
    assert rel_max(got, ref, cells) <= 1e-6


def test_product_smoother_reduces_the_residual(adaptive):
    c = adaptive
    b = c.rand(12)
    x0 = np.zeros_like(b)
    r0 = np.linalg.norm(c.ctx.residual(0, x0, b))
    x = x0
    for k in range(3):
        x = c.ctx.relax(0, x, b, 1, k & 1, inner=3, mode=0)
        r = np.linalg.norm(c.ctx.residual(0, x, b))
        assert r < r0
        r0 = r


def test_vcycle_is_linear_symmetric_and_contracting(adaptive):
    """The V-cycle preconditioner z = V r: linear, symmetric (<r1, V r2> =
    <r2, V r1>, the post-smoother is the pre-smoother's adjoint), positive,
    and its error in the energy norm below that of z = 0 for A e = r, e from
    the FP64 oracle."""
    c = adaptive
    r1, r2 = c.rand(13).astype(np.float64), c.rand(14).astype(np.float64)
    z1, z2 = c.ctx.vcycle(r1), c.ctx.vcycle(r2)
    z12 = c.ctx.vcycle(0.5 * r1 - 2.0 * r2)
    assert rel_max(z12, 0.5 * z1 - 2.0 * z2) <= 1e-5
    s12, s21 = float(r1 @ z2), float(r2 @ z1)
    assert abs(s12 - s21) <= 1e-5 * np.sqrt(abs(float(r1 @ z1) * float(r2 @ z2)))
    assert float(r1 @ z1) > 0 and float(r2 @ z2) > 0
    def apply(v):  # the oracle's operator on the scene the GPU prepared
        return oracle.pressure_apply_oracle(c.scene, v)

    # e = A^-1 r1: Jacobi-preconditioned CG in FP64 on the oracle operator
    diag = c.ctx.diagonal(0).astype(np.float64)
    inv = np.where(diag > 0, 1.0 / np.maximum(diag, 1e-300), 0.0)
    e = np.zeros_like(r1)
    res = r1.copy()
    zz = inv * res
    d = zz.copy()
    rho = res @ zz
    for _ in range(4000):
        q = apply(d)
        al = rho / (d @ q)
        e += al * d
        res -= al * q
        if np.linalg.norm(res) <= 1e-10 * np.linalg.norm(r1):
            break
        zz = inv * res
        rn = res @ zz
        d = zz + (rn / rho) * d
        rho = rn
    assert np.linalg.norm(res) <= 1e-10 * np.linalg.norm(r1)
    err_v = e - z1
    assert float(err_v @ apply(err_v)) < 0.5 * float(e @ apply(e))
