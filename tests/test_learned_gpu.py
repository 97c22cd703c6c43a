"""Ablation of the learned initial guess inside the pressure solve.

A network is trained on the GPU (the library's own forward, backward and Adam
kernels) on (right-hand side, solution) tile pairs that the refined solver
produces on seeded sphere-union instances, then used as the initial guess of
the refined MGPCG on an unseen instance.  The test states what it gains over
the same solve without it: the energy-norm error of the starting iterate
(against the FP64 oracle) and the PCG iterations; plain MGPCG stays the judge
(the learned solve must still reach the true residual 1e-6 and the oracle's
solution within 1e-5)."""
import numpy as np
import pytest

import msbg_gpu
import oracle

pytestmark = pytest.mark.gpu


def scene(seed):
    # sphere-union liquid, Fourier-mode RHS, 32^3 base blocks, 2 levels
    return msbg_gpu.PressureScene(128, 32, 2, 0.0, 24, 0.08, 0.2, 4, 16, 8, 8.0, seed)


def energy(s, e):
    return float(e @ oracle.pressure_apply_oracle(s, e))


@pytest.fixture(scope="module")
def trained():
    import torch
    ctx = msbg_gpu.Context(0)
    F, T, M = [], [], []
    for seed in range(6):
        ctx.pressure_prepare(scene(300 + seed))
        info = ctx.pressure_solve(tol=1e-6, maxRefine=4)
        assert info.status == 0
        f, t, m = msbg_gpu.collect_training_pairs(ctx, 400)
        F.append(f)
        T.append(t)
        M.append(m)
    F, T, M = torch.cat(F), torch.cat(T), torch.cat(M)
    net = msbg_gpu.Cnn(0)
    losses = msbg_gpu.train_cnn(net, F, T, M, epochs=30, batch=64, lr=2e-3, seed=3)
    yield ctx, net, losses
    ctx.close()
    net.close()


def test_training_loss_decreases(trained):
    _, _, losses = trained
    assert losses[-1] < 0.8 * losses[0], losses


def test_learned_guess_gains_over_zero_guess(trained):
    ctx, net, _ = trained
    s = scene(999)  # unseen instance
    ctx.pressure_prepare(s)
    ctx.pressure_set_cnn(net)
    plain = ctx.pressure_solve(tol=1e-6, maxRefine=30)
    learned = ctx.pressure_solve(tol=1e-6, maxRefine=30, learned=1)
    x = ctx.pressure_download(fp64=True)
    xo, bo, _, _ = oracle.pressure_oracle(s, tol=1e-12)
    # the learned solve is still judged by plain MGPCG's criteria
    assert learned.status == 0 and learned.relResidual <= 1e-6
    assert np.linalg.norm(x - xo) <= 1e-5 * np.linalg.norm(xo)
    # what the network gains: a starting iterate closer in the energy norm
    g = ctx.pressure_learned_guess().astype(np.float64)
    e0, eg = energy(s, xo), energy(s, g - xo)
    untrained = msbg_gpu.Cnn(0)
    ctx.pressure_set_cnn(untrained)
    eu = energy(s, ctx.pressure_learned_guess().astype(np.float64) - xo)
    ctx.pressure_set_cnn(net)
    print(f"energy error of x0: zero 1, trained {eg / e0:.3f}, untrained {eu / e0:.3f}; "
          f"PCG iterations: plain {plain.iterations}, learned {learned.iterations}")
    assert eg < 0.9 * e0
    assert eg < eu
    assert learned.iterations <= plain.iterations
    untrained.close()
