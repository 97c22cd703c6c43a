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


VCYCLE = dict(nPre=2, nPost=2, innerIter=3)


@pytest.fixture(scope="module")
def trained():
    """The guess network (right-hand side -> solution) and the correction
    network (residual after a V-cycle -> error after it), each trained on
    pairs from six seeded instances."""
    import torch
    ctx = msbg_gpu.Context(0)
    G, K = [], []
    for seed in range(6):
        ctx.pressure_prepare(scene(300 + seed))
        info = ctx.pressure_solve(tol=1e-6, maxRefine=4)
        assert info.status == 0
        G.append(msbg_gpu.collect_training_pairs(ctx, 400))
        for k in (0, 1, 2):
            K.append(msbg_gpu.collect_correction_pairs(ctx, 150, k, **VCYCLE))
    cat = lambda P: [torch.cat([q[j] for q in P]) for j in range(3)]
    net = msbg_gpu.Cnn(0)
    losses = msbg_gpu.train_cnn(net, *cat(G), epochs=30, batch=64, lr=2e-3, seed=3)
    corr = msbg_gpu.Cnn(0)
    closs = msbg_gpu.train_cnn(corr, *cat(K), epochs=30, batch=64, lr=2e-3, seed=4)
    yield ctx, net, losses, corr, closs
    ctx.close()
    net.close()
    corr.close()


def test_training_loss_decreases(trained):
    _, _, losses, _, closs = trained
    assert losses[-1] < 0.8 * losses[0], losses
    assert closs[-1] < 0.9 * closs[0], closs


def test_learned_guess_gains_over_zero_guess(trained):
    ctx, net, _, _, _ = trained
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


def masked_rel_err(pred, target, mask):
    return float((((pred - target) ** 2) * mask).sum() / ((target ** 2) * mask).sum()) ** 0.5


def test_correction_network_gains_on_unseen_instance(trained):
    """What the correction network gains: on an unseen instance, its estimate
    of the error a V-cycle leaves (inside PCG, after 1 iteration) is closer
    to that error than zero (the V-cycle alone) and than an untrained
    network's estimate."""
    ctx, _, _, corr, _ = trained
    ctx.pressure_prepare(scene(996))
    assert ctx.pressure_solve(tol=1e-6, maxRefine=4).status == 0
    f, t, m = msbg_gpu.collect_correction_pairs(ctx, 300, 1, **VCYCLE)
    untrained = msbg_gpu.Cnn(0)
    et = masked_rel_err(corr.forward(f), t, m)
    eu = masked_rel_err(untrained.forward(f), t, m)
    untrained.close()
    print(f"relative error of the V-cycle's leftover estimate: zero 1, trained {et:.3f}, "
          f"untrained {eu:.3f}")
    assert et < 1.0 and et < eu


@pytest.mark.parametrize("mode", [2, 3])
def test_learned_correction_flexible_cg(trained, mode):
    """learned bit 1: the correction network also corrects every V-cycle
    (z = V r + omega net(r - A V r)) under flexible CG; with bit 0 the guess
    network starts it.  It meets plain MGPCG's criteria, and with the
    energy-optimal omega an untrained network cannot derail it."""
    ctx, net, _, corr, _ = trained
    s = scene(998)
    ctx.pressure_prepare(s)
    ctx.pressure_set_cnn(net)
    xo, _, _, _ = oracle.pressure_oracle(s, tol=1e-12)
    plain = ctx.pressure_solve(tol=1e-6, maxRefine=30, **VCYCLE)
    untrained = msbg_gpu.Cnn(0)
    for which in (corr, untrained):
        ctx.pressure_set_correction_cnn(which)
        info = ctx.pressure_solve(tol=1e-6, maxRefine=30, learned=mode, **VCYCLE)
        x = ctx.pressure_download(fp64=True)
        print(f"learned={mode} {'trained' if which is corr else 'untrained'}: iterations "
              f"{info.iterations} (plain {plain.iterations})")
        assert info.status == 0 and info.relResidual <= 1e-6 and info.learnedFallback == 0
        assert np.linalg.norm(x - xo) <= 1e-5 * np.linalg.norm(xo)
        assert info.iterations <= plain.iterations + 2
    ctx.pressure_set_correction_cnn(corr)
    untrained.close()
    with pytest.raises(msbg_gpu.MsbgError):
        ctx.pressure_solve(tol=1e-6, storage=msbg_gpu.F16, learned=2)


@pytest.mark.parametrize("mode", [1, 2])
def test_plain_mgpcg_is_the_fallback(trained, mode):
    """A network whose output is not finite makes the learned solve stop
    (status 3); the solve then falls back to plain MGPCG from zero and still
    delivers the 1e-6 solution, reporting the fallback."""
    ctx, net, _, corr, _ = trained
    s = scene(997)
    ctx.pressure_prepare(s)
    bad = msbg_gpu.Cnn(0)
    bad.set_weights(np.full(bad.n_params, np.nan, np.float32))
    (ctx.pressure_set_cnn if mode == 1 else ctx.pressure_set_correction_cnn)(bad)
    info = ctx.pressure_solve(tol=1e-6, maxRefine=30, learned=mode)
    ctx.pressure_set_cnn(net)
    ctx.pressure_set_correction_cnn(corr)
    bad.close()
    assert info.learnedFallback == 1
    assert info.status == 0 and info.relResidual <= 1e-6
    xo, _, _, _ = oracle.pressure_oracle(s, tol=1e-12)
    x = ctx.pressure_download(fp64=True)
    assert np.linalg.norm(x - xo) <= 1e-5 * np.linalg.norm(xo)
    good = ctx.pressure_solve(tol=1e-6, maxRefine=30, learned=mode)
    assert good.learnedFallback == 0 and good.status == 0
