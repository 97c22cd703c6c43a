"""The CPU restatement of the FLIP transfers (oracle/msbg_oracle_flip.c,
following src/flip_sim.cpp) on properties the reference's code has by
construction: P2G conserves the particle count in the cell masses and
reproduces a uniform particle velocity on every weighted face; G2P returns a
uniform grid velocity; the gradient update with p = 0 only clears the faces
without liquid and the lower domain faces; gravity adds g dt next to liquid."""
import numpy as np

import msbg_gpu
import oracle

RES, BSX = 32, 16


def particles():
    return msbg_gpu.flip_particles(RES, BSX, z_liquid=0.4, ppv=8, air_ppv=1, seed=3)


def test_p2g_mass_and_uniform_velocity():
    p = particles()
    p["vel"] = np.array([1.0, -2.0, 0.5], np.float32)
    vel, mass, beta, act = oracle.flip_p2g(RES, BSX, p)
    assert mass.sum() == len(p)
    v = vel.reshape(-1, 3)
    # faces with weight hold the particles' velocity
    for d, u in enumerate((1.0, -2.0, 0.5)):
        nz = v[:, d] != 0
        assert nz.sum() > 0 and np.allclose(v[nz, d], u, rtol=1e-6)
    assert act.sum() >= 1 and ((beta > 0) & (beta <= 1.0)).all()


def test_g2p_returns_a_uniform_grid_velocity_inside():
    p = particles()
    n = RES ** 3
    vel = np.tile(np.array([0.25, 0.5, -1.0], np.float32), n)
    q = oracle.flip_g2p(RES, BSX, p, vel, vel, 0.0)  # pure PIC
    inside = ((p["pos"] > 1.0) & (p["pos"] < RES - 1.0)).all(1)
    assert np.allclose(q["vel"][inside], [0.25, 0.5, -1.0], rtol=1e-6)


def test_gradient_with_zero_pressure_and_gravity():
    p = particles()
    vel, mass, beta, _ = oracle.flip_p2g(RES, BSX, p)
    v2 = oracle.flip_gradient(RES, BSX, vel, mass, beta, np.zeros(RES ** 3, np.float32), 0.01)
    changed = v2 != vel
    assert (v2[changed] == 0).all()
    g, old = oracle.flip_gravity(RES, BSX, vel, mass, -9.8, 0.1)
    assert np.array_equal(old, vel)
    dv = (g - vel).reshape(-1, 3)
    assert np.isclose(dv[:, 1], -0.98).any() and (np.abs(dv[:, [0, 2]]) <= np.abs(
        vel.reshape(-1, 3)[:, [0, 2]]) + 1e-7).all()
