"""FP64 CPU oracle of the learned 3D CNN (test infrastructure only).

The network has no counterpart in the reference (it is one of the solver's
additions); this file restates its mathematics in numpy float64 so that the
GPU kernels (msbg-flip_b200/csrc/cnn.cu) can be checked against it:

  conv1 4->16 valid on the 18^3 box, ReLU; conv2, conv3 16->16 with zero
  padding, ReLU; conv4 16->1 with zero padding; 3^3 kernels, no biases;
  weights per layer in [cout][cin][kz][ky][kx] order (cross-correlation, as
  torch.nn.Conv3d).  Loss = sum(mask * (y - target)^2) / count.

With quant=True the oracle rounds to BF16 (round to nearest even) exactly
where the GPU stores BF16: the weights, the input features, the post-ReLU
activations, dL/dy and the masked data gradients; everything else is FP64.
Its own backward pass is pinned by central finite differences in
tests/test_cnn_oracle.py.
"""
from __future__ import annotations

import numpy as np

NFEAT, NC, TS, PD = 4, 16, 16, 18
LAYERS = [(NFEAT, NC), (NC, NC), (NC, NC), (NC, 1)]  # (cin, cout)
NPARAM = sum(27 * ci * co for ci, co in LAYERS)


def bf16(x):
    """Round float values to bfloat16 (nearest even), returned as float64."""
    x32 = np.ascontiguousarray(x, dtype=np.float32)
    u = x32.view(np.uint32).astype(np.uint64)
    r = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    return r.astype(np.uint32).view(np.float32).astype(np.float64)


def split_weights(w):
    """Flat FP32/FP64 weights -> list of [cout][cin][3][3][3] arrays."""
    out, o = [], 0
    for ci, co in LAYERS:
        n = 27 * ci * co
        out.append(np.asarray(w[o:o + n], np.float64).reshape(co, ci, 3, 3, 3))
        o += n
    return out


def conv_valid(W, X):
    """out[co, z, y, x] = sum_{ci,k} W[co, ci, k] X[ci, z+kz, y+ky, x+kx] on an 18^3 box."""
    out = np.zeros((W.shape[0], TS, TS, TS))
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                out += np.einsum('oc,czyx->ozyx', W[:, :, kz, ky, kx],
                                 X[:, kz:kz + TS, ky:ky + TS, kx:kx + TS], optimize=True)
    return out


def pad(A):
    return np.pad(A, ((0, 0), (1, 1), (1, 1), (1, 1)))


def flip_t(W):
    """Kernel of the data gradient: W'[ci][co][k] = W[co][ci][2 - k]."""
    return np.ascontiguousarray(W[:, :, ::-1, ::-1, ::-1].transpose(1, 0, 2, 3, 4))


def wgrad(dZ, Xp):
    """dW[co, ci, k] = sum_o dZ[co, o] Xp[ci, o + k]."""
    g = np.zeros((dZ.shape[0], Xp.shape[0], 3, 3, 3))
    for kz in range(3):
        for ky in range(3):
            for kx in range(3):
                g[:, :, kz, ky, kx] = np.einsum('ozyx,czyx->oc', dZ,
                                                Xp[:, kz:kz + TS, ky:ky + TS, kx:kx + TS],
                                                optimize=True)
    return g


def forward(w, feat, quant=True):
    """feat [4][18][18][18] -> (y [16][16][16], saved activations)."""
    q = bf16 if quant else (lambda a: np.asarray(a, np.float64))
    W = [q(Wl) for Wl in split_weights(w)]
    x0 = q(feat)
    a1 = q(np.maximum(conv_valid(W[0], x0), 0))
    a2 = q(np.maximum(conv_valid(W[1], pad(a1)), 0))
    a3 = q(np.maximum(conv_valid(W[2], pad(a2)), 0))
    y = conv_valid(W[3], pad(a3))[0]
    return y, (W, x0, a1, a2, a3)


def loss_grad(w, feats, targets, masks, count, quant=True):
    """Loss and FP64 gradient (flat, the weight layout) over a batch of tiles."""
    q = bf16 if quant else (lambda a: np.asarray(a, np.float64))
    grads = [np.zeros((co, ci, 3, 3, 3)) for ci, co in LAYERS]
    loss = 0.0
    for f, t, m in zip(feats, targets, masks):
        y, (W, x0, a1, a2, a3) = forward(w, f, quant)
        d = np.where(m > 0, y - t, 0.0)
        loss += float((d * d).sum()) / count
        dy = q(2.0 * d / count)[None]
        dz3 = q(conv_valid(flip_t(W[3]), pad(dy)) * (a3 > 0))
        dz2 = q(conv_valid(flip_t(W[2]), pad(dz3)) * (a2 > 0))
        dz1 = q(conv_valid(flip_t(W[1]), pad(dz2)) * (a1 > 0))
        grads[3] += wgrad(dy, pad(a3))
        grads[2] += wgrad(dz3, pad(a2))
        grads[1] += wgrad(dz2, pad(a1))
        grads[0] += wgrad(dz1, x0)
    return loss, np.concatenate([g.ravel() for g in grads])
