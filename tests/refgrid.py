"""Helpers of the pressure parity tests against the compiled reference.

Grids: the reference's pressure path needs at least 2 resolution levels
(MultiresSparseGrid with nLevels = 1 exits in its prepare), so a
"single-level" grid here is nLevels = 2 with every block at level 0, and an
adaptive grid is nLevels = 2 with a narrow fine band.  Base blocks are 16^3:
the reference's smoother aborts for 32^3 blocks (src/msbg3.cpp:1692-1749).
"""
import numpy as np

# (res, bsx0, nLevels, band): every block at level 0 / adaptive 2-level map
SINGLE = (64, 16, 2, 8.0)
ADAPTIVE = (128, 16, 2, 4.0)


def block_offsets(block_levels, bsx0):
    sizes = [(bsx0 >> int(l)) ** 3 for l in block_levels]
    return np.concatenate([[0], np.cumsum(sizes)]).astype(np.int64)


def cell_levels(block_levels, bsx0):
    return np.repeat(np.asarray(block_levels), [(bsx0 >> int(l)) ** 3 for l in block_levels])


def interface_mask(block_levels, res, bsx0):
    """True for the cells of a block face whose neighbour block has another
    resolution level: the cells where the reference's operator (mixed-level
    ghosts, src/msbg3.cpp:46-161, and its diagonal, src/msbg3.cpp:2686-2731)
    and the finite-volume operator differ by design."""
    nb1 = res // bsx0
    bl = np.asarray(block_levels)
    out = []
    for b, l in enumerate(bl):
        bx, by, bz = b % nb1, (b // nb1) % nb1, b // (nb1 * nb1)
        bs = bsx0 >> int(l)
        m = np.zeros((bs, bs, bs), bool)  # [z, y, x]
        for dx, dy, dz in ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)):
            X, Y, Z = bx + dx, by + dy, bz + dz
            if not (0 <= X < nb1 and 0 <= Y < nb1 and 0 <= Z < nb1):
                continue
            if bl[X + nb1 * (Y + nb1 * Z)] == l:
                continue
            if dx:
                m[:, :, 0 if dx < 0 else -1] = True
            if dy:
                m[:, 0 if dy < 0 else -1, :] = True
            if dz:
                m[0 if dz < 0 else -1, :, :] = True
        out.append(m.ravel())
    return np.concatenate(out)


def blocks_without_interface(block_levels, res, bsx0):
    """Per block: True when none of its six face neighbours has another level."""
    nb1 = res // bsx0
    bl = np.asarray(block_levels)
    ok = np.ones(len(bl), bool)
    for b, l in enumerate(bl):
        bx, by, bz = b % nb1, (b // nb1) % nb1, b // (nb1 * nb1)
        for dx, dy, dz in ((-1, 0, 0), (1, 0, 0), (0, -1, 0), (0, 1, 0), (0, 0, -1), (0, 0, 1)):
            X, Y, Z = bx + dx, by + dy, bz + dz
            if 0 <= X < nb1 and 0 <= Y < nb1 and 0 <= Z < nb1 and bl[X + nb1 * (Y + nb1 * Z)] != l:
                ok[b] = False
    return ok


def block_parity(res, bsx0):
    nb1 = res // bsx0
    b = np.arange(nb1 ** 3)
    return (b % nb1 + (b // nb1) % nb1 + b // (nb1 * nb1)) & 1


def rel_max(a, ref, mask=None):
    """max |a - ref| / max |ref| over the masked cells."""
    if mask is not None:
        a, ref = a[mask], ref[mask]
    s = float(np.abs(ref).max())
    return float(np.abs(a - ref).max()) / (s if s > 0 else 1.0)


def to_blocks(dense, bsx0):
    """Dense [z, y, x] array of a grid with every block at level 0 -> the
    packed block layout (blocks in bid order, vid = x + y*bs + z*bs*bs)."""
    nz, ny, nx = dense.shape
    v = dense.reshape(nz // bsx0, bsx0, ny // bsx0, bsx0, nx // bsx0, bsx0)
    return np.ascontiguousarray(v.transpose(0, 2, 4, 1, 3, 5)).reshape(-1)


def box_problem(res=32, bsx0=16, z_liquid=20, seed=0):
    """A liquid pool (z < z_liquid) under air in a box with solid walls, every
    block at level 0, as per-cell arrays: (flags, [faceX, faceY, faceZ], rhs)
    in the packed block layout.  Face coefficients are 1, and 0 on the lower
    domain faces (the upper ones lie outside the arrays and read 0)."""
    z, y, x = np.meshgrid(np.arange(res), np.arange(res), np.arange(res), indexing="ij")
    flags = np.where(z < z_liquid, 0, 0x1000).astype(np.uint16)
    faces = []
    for d, c in enumerate((x, y, z)):
        f = np.ones((res,) * 3, np.float32)
        f[c == 0] = 0.0
        faces.append(f)
    rng = np.random.default_rng(seed)
    rhs = (rng.standard_normal((res,) * 3) * (z < z_liquid)).astype(np.float32)
    return (to_blocks(flags, bsx0), [to_blocks(f, bsx0) for f in faces], to_blocks(rhs, bsx0))


class OpenPool:
    """A pool (liquid below z = z_liquid, air above) on a grid with every
    block at level 0 whose face callback returns `face` for every face,
    inside the grid or not, so that each domain-face rule shows in A x.  Has
    the interface of msbg_gpu.PressureScene that the oracle functions and the
    reference driver read."""

    def __init__(self, res=16, bsx0=16, z_liquid=12, face=0.5):
        import ctypes as C

        import msbg_gpu

        self.res, self.bsx0, self.n_levels = res, bsx0, 2
        self.block_levels = np.zeros((res // bsx0) ** 3, np.int32)
        self._ct = C.CFUNCTYPE(C.c_uint16, C.c_void_p, C.c_int, C.c_int, C.c_int)(
            lambda u, x, y, z: 0 if z < z_liquid else 0x1000)
        self._fc = C.CFUNCTYPE(C.c_float, C.c_void_p, C.c_int, C.c_int, C.c_int, C.c_int)(
            lambda u, d, x, y, z: face)
        self._rh = C.CFUNCTYPE(C.c_float, C.c_void_p, C.c_int, C.c_int, C.c_int)(
            lambda u, x, y, z: 1.0)
        self._cb = msbg_gpu.PressureCallbacks(C.cast(self._ct, C.c_void_p).value,
                                              C.cast(self._fc, C.c_void_p).value,
                                              C.cast(self._rh, C.c_void_p).value, None)

    def callbacks(self):
        return self._cb

    def packed_size(self):
        return self.res ** 3
