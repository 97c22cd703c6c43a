"""The learned network's tensor-core kernels against the FP64 oracle.

Forward outputs and weight gradients of the GPU network (tcgen05 implicit-GEMM
convolutions, BF16 operands, FP32 accumulation) are compared with
oracle/cnn_oracle.py run with BF16 rounding at the same points; what is left
is FP32-vs-FP64 summation order and rare BF16 rounding-boundary flips, so the
bound is 5e-3 (forward) and 1e-2 (gradients) in relative norm."""
import numpy as np
import pytest

import cnn_oracle as co
import msbg_gpu

pytestmark = pytest.mark.gpu


def rel(a, b):
    return float(np.linalg.norm(a - b) / max(1e-300, np.linalg.norm(b)))


def case(seed, n):
    rng = np.random.default_rng(seed)
    w = np.concatenate([rng.uniform(-1, 1, 27 * ci * cout) * np.sqrt(6.0 / (27 * ci))
                        for ci, cout in co.LAYERS]).astype(np.float32)
    feat = rng.standard_normal((n, 4, 18, 18, 18)).astype(np.float32)
    feat[:, 1:3] = (feat[:, 1:3] > 0.5)  # mask-like channels
    feat[:, 3] = 0.5
    tgt = rng.standard_normal((n, 16, 16, 16)).astype(np.float32)
    mask = (rng.random((n, 16, 16, 16)) < 0.8).astype(np.float32)
    return w, feat, tgt, mask


def to_dev(a):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a).reshape(a.shape[0], -1)).cuda()


def test_forward_matches_oracle():
    w, feat, _, _ = case(1, 3)
    net = msbg_gpu.Cnn(0)
    net.set_weights(w)
    y = net.forward(to_dev(feat)).cpu().numpy().reshape(3, 16, 16, 16)
    for t in range(3):
        yo, _ = co.forward(w.astype(np.float64), feat[t], quant=True)
        assert rel(y[t], yo) <= 5e-3, (t, rel(y[t], yo))
        ye, _ = co.forward(w.astype(np.float64), feat[t], quant=False)
        assert rel(y[t], ye) <= 3e-2
    net.close()


def test_weight_gradients_match_oracle():
    w, feat, tgt, mask = case(2, 3)
    net = msbg_gpu.Cnn(0)
    net.set_weights(w)
    count = float(mask.sum())
    loss, g = net.loss_grad(to_dev(feat), to_dev(tgt), to_dev(mask), count=count, want_grad=True)
    lo, go = co.loss_grad(w.astype(np.float64), list(feat), list(tgt), list(mask), count,
                          quant=True)
    assert abs(loss - lo) <= 5e-3 * abs(lo)
    offs = np.cumsum([0] + [27 * ci * cout for ci, cout in co.LAYERS])
    for l in range(4):
        e = rel(g[offs[l]:offs[l + 1]], go[offs[l]:offs[l + 1]])
        assert e <= 1e-2, (l, e)
    net.close()


def test_training_on_the_gpu_fits_a_teacher_network():
    """The GPU trainer (own forward, backward and Adam kernels) fits targets
    made by a random teacher network of the same shape."""
    import torch
    rng = np.random.default_rng(4)
    n = 48
    _, feat, _, _ = case(5, n)
    teacher = msbg_gpu.Cnn(0)
    wt, _, _, _ = case(6, 1)
    teacher.set_weights(wt)
    fd = to_dev(feat)
    tgt = teacher.forward(fd)
    mask = torch.ones_like(tgt)
    student = msbg_gpu.Cnn(0)
    l0 = student.loss_grad(fd, tgt, mask)
    losses = msbg_gpu.train_cnn(student, fd, tgt, mask, epochs=30, batch=16, lr=3e-3, seed=1)
    assert losses[-1] < 0.2 * l0, (l0, losses[-1])
    teacher.close()
    student.close()


def test_forward_is_deterministic():
    w, feat, _, _ = case(7, 5)
    net = msbg_gpu.Cnn(0)
    net.set_weights(w)
    a = net.forward(to_dev(feat)).cpu().numpy()
    b = net.forward(to_dev(feat)).cpu().numpy()
    np.testing.assert_array_equal(a, b)
    net.close()
