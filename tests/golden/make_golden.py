"""Generate the golden fixtures of the smoother from the compiled reference.

Runs the unmodified reference MultiresSparseGrid::applyChannelPdeFast<float>
(MCF, 8-colour) through oracle/_ref/libmsbg_ref.so (built from the reference
sources by oracle/Makefile) on small seeded grids and stores inputs and
outputs as .npz files beside this script.  Re-run with
``python tests/golden/make_golden.py`` (needs the reference tree to build the
library; the fixtures themselves travel without it).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402


def smooth_field(rng, res3, bsx, kind):
    """A smooth random field (sum of a few sinusoids) cut into value blocks."""
    sx, sy, sz = res3
    z, y, x = np.meshgrid(np.arange(sz), np.arange(sy), np.arange(sx), indexing="ij")
    f = np.zeros((sz, sy, sx), np.float64)
    for _ in range(6):
        k = rng.uniform(0.05, 0.3, 3)
        f += rng.normal() * 3 * np.sin(k[0] * x + k[1] * y + k[2] * z + rng.uniform(0, 6.3))
    f += 0.2 * (x - sx / 2)  # non-zero gradient almost everywhere
    nbx, nby, nbz = sx // bsx, sy // bsx, sz // bsx
    blocks = []
    for bid in range(len(kind)):
        if kind[bid] != 1:
            continue
        bx, by, bz = bid % nbx, (bid // nbx) % nby, bid // (nbx * nby)
        blocks.append(f[bz * bsx:(bz + 1) * bsx, by * bsx:(by + 1) * bsx, bx * bsx:(bx + 1) * bsx])
    return np.stack(blocks).astype(np.float32)


CASES = {
    # name: (res3, bsx, seed, kind probabilities [null, value, empty, full], update fraction, clamp01)
    "mcf_value_const_null_b8": ((32, 32, 32), 8, 11, [0.15, 0.6, 0.15, 0.1], 0.85, False),
    "mcf_aniso_b16": ((64, 32, 32), 16, 12, [0.1, 0.7, 0.1, 0.1], 1.0, False),
    "mcf_clamp01_b8": ((24, 16, 32), 8, 13, [0.0, 1.0, 0.0, 0.0], 1.0, True),
}


def make(name, res3, bsx, seed, probs, frac, clamp01):
    rng = np.random.default_rng(seed)
    nb = (res3[0] // bsx) * (res3[1] // bsx) * (res3[2] // bsx)
    kind = rng.choice(4, size=nb, p=probs).astype(np.int8)
    if not (kind == 1).any():
        kind[0] = 1
    vals = smooth_field(rng, res3, bsx, kind)
    if clamp01:
        vals = (0.5 + 0.05 * vals).astype(np.float32)
    ids = np.nonzero(kind == 1)[0]
    upd = np.sort(rng.choice(ids, size=max(1, int(round(frac * len(ids)))), replace=False))
    upd = upd.astype(np.int32)
    ev, fv = (1.0, 0.0) if clamp01 else (4.0, -4.0)
    out2, _ = oracle.mcf_reference(res3, bsx, kind, vals, upd, 2, 0.1, clamp01, ev, fv)
    out20, _ = oracle.mcf_reference(res3, bsx, kind, vals, upd, 20, 0.1, clamp01, ev, fv)
    np.savez_compressed(os.path.join(HERE, name + ".npz"), res3=np.array(res3), bsx=bsx,
                        kind=kind, values=vals, update=upd, dt=np.float32(0.1),
                        clamp01=int(clamp01), empty_val=np.float32(ev), full_val=np.float32(fv),
                        out2=out2, out20=out20)
    print(name, "blocks", nb, "value", len(ids), "updated", len(upd))


if __name__ == "__main__":
    if not oracle.ref_available():
        oracle.build_ref()
    for n, c in CASES.items():
        make(n, *c)
