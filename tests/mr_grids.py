"""Seeded mixed-resolution block-level maps and particles shared by the tests of
G2P on grids with several levels.  Every map keeps 26-neighbour blocks within
one level of each other, as the reference requires (src/msbg.cpp:1718-1719)."""
import numpy as np

# name: (res, bsx0, nLevels, kind)
GRIDS = {
    "z3_b16": (128, 16, 3, "z"),       # levels in z slabs: 0 below, 1, 2 on top
    "sphere2_b8": (64, 8, 2, "sphere"),  # level 0 inside a sphere, 1 outside
    "z2_b32": (128, 32, 2, "z"),
    "sphere3_b16": (128, 16, 3, "sphere"),
}


def grid_levels(name):
    res, bsx, nl, kind = GRIDS[name]
    nb = res // bsx
    b = np.arange(nb ** 3)
    bx, by, bz = b % nb, (b // nb) % nb, b // (nb * nb)
    if kind == "z":
        lev = np.where(bz < nb * 3 // 8, 0, np.where(bz < nb * 6 // 8, 1, 2))
    else:
        # level shells 2 blocks apart: neighbours (at most sqrt(3) apart)
        # never skip a level
        r = np.sqrt((bx - nb / 2 + .5) ** 2 + (by - nb / 2 + .5) ** 2 + (bz - nb / 2 + .5) ** 2)
        lev = np.where(r < nb / 5, 0, np.where(r < nb / 5 + 2, 1, 2))
    return res, bsx, nl, np.minimum(lev, nl - 1).astype(np.int32)


def particles_for(res, n, seed, margin=1.5, n_nan=16):
    """n seeded particles over the grid and margin voxels beyond it, a few on
    voxel corners and faces, n_nan with a non-finite position."""
    import msbg_gpu

    rng = np.random.default_rng(seed)
    p = np.zeros(n, msbg_gpu.FLIP_PARTICLE)
    pos = rng.uniform(-margin, res + margin, (n, 3)).astype(np.float32)
    pos[: n // 20] = np.round(pos[: n // 20] * 2) / 2
    p["pos"] = pos
    p["vel"] = rng.standard_normal((n, 3)).astype(np.float32)
    p["pos"][n // 2: n // 2 + n_nan, n_nan % 3] = np.nan
    return p
