"""CPU tests of the learned network's FP64 oracle (oracle/cnn_oracle.py).

The network has no counterpart in the reference, so the oracle is pinned by
mathematics: its backward pass against central finite differences of its own
forward pass (FP64, no BF16 rounding), and its BF16 rounding against torch's
float32 -> bfloat16 conversion."""
import numpy as np
import pytest

import cnn_oracle as co


def random_case(seed, n=1):
    rng = np.random.default_rng(seed)
    w = np.concatenate([rng.uniform(-1, 1, 27 * ci * cout) * np.sqrt(6.0 / (27 * ci))
                        for ci, cout in co.LAYERS])
    feats = [rng.standard_normal((4, 18, 18, 18)) for _ in range(n)]
    targets = [rng.standard_normal((16, 16, 16)) for _ in range(n)]
    masks = [(rng.random((16, 16, 16)) < 0.7).astype(np.float64) for _ in range(n)]
    return w, feats, targets, masks


def test_oracle_gradient_matches_finite_differences():
    w, f, t, m = random_case(3)
    count = float(sum(x.sum() for x in m))
    loss, g = co.loss_grad(w, f, t, m, count, quant=False)
    assert g.shape == (co.NPARAM,)
    rng = np.random.default_rng(7)
    offs = np.cumsum([0] + [27 * ci * cout for ci, cout in co.LAYERS])
    idx = [int(rng.integers(offs[l], offs[l + 1])) for l in range(4) for _ in range(3)]
    h = 1e-6
    for i in idx:
        wp, wm = w.copy(), w.copy()
        wp[i] += h
        wm[i] -= h
        lp, _ = co.loss_grad(wp, f, t, m, count, quant=False)
        lm, _ = co.loss_grad(wm, f, t, m, count, quant=False)
        fd = (lp - lm) / (2 * h)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)), (i, fd, g[i])


def test_bf16_rounding_matches_torch():
    torch = pytest.importorskip("torch")
    x = np.random.default_rng(1).standard_normal(100000).astype(np.float32) * 10.0
    ref = torch.from_numpy(x).to(torch.bfloat16).to(torch.float64).numpy()
    np.testing.assert_array_equal(co.bf16(x), ref)


def test_quantised_and_exact_oracles_agree_to_bf16_precision():
    w, f, t, m = random_case(5)
    yq, _ = co.forward(w, f[0], quant=True)
    ye, _ = co.forward(w, f[0], quant=False)
    assert np.linalg.norm(yq - ye) <= 3e-2 * np.linalg.norm(ye)
