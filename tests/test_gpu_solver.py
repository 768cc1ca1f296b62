"""The GPU basic scheme against the oracle, per iterate, and the tutorial's
published effective stiffness (square_basic.rst:227)."""
import numpy as np
import pytest
import torch

import janus_b200.material.elastic.linear.isotropic as material
from janus_b200 import microstructures as micro
from janus_b200 import operators as ops
from janus_b200.green import filtered, truncated
from janus_b200.solvers import BasicScheme
from oracle import janus_oracle as O

FACTORY = {"truncated": truncated, "filtered": filtered}


def _problem(phase, mats, g0, nu0, variant, dtype=None):
    dim = phase.ndim
    pars = [O.delta_c(g, nu, g0, nu0, dim) for g, nu in mats]
    tens = [ops.isotropic_4(s, d, dim) for s, d in pars]
    cls = ops.BlockDiagonalOperator2D if dim == 2 else ops.BlockDiagonalOperator3D
    loc = cls.from_phases(phase, tens, dtype=dtype)
    green = FACTORY[variant](material.create(g0, nu0, dim).green_operator(), phase.shape, 1.0,
                             dtype=dtype)
    return loc, green, [p[0] for p in pars], [p[1] for p in pars]


@pytest.mark.gpu
def test_tutorial_effective_stiffness():
    # square_basic.py:60-97: corner square, mu_0 = 50, nu_i = 0.2, 400 its
    phase = micro.square_inclusion(256, centered=False)
    loc, green, _, _ = _problem(phase, [(1.0, 0.3), (100.0, 0.2)], 50.0, 0.3, "truncated")
    E = np.array([0., 0., 1.])
    r = BasicScheme(green, loc).run(E, 400)
    c1212 = 50.0 + 0.5 * r.mean_tau[0, -1] / E[-1]
    assert abs(c1212 - 1.41903971282) < 5e-12
    assert r.iterations == 400


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
def test_square_inclusion_per_iterate(variant):
    """Config 1: 256^2 centred square (side 128), mu 1/100, mu_0 = 50.5,
    200 iterations; every checked iterate within 1e-12 of the oracle."""
    n = 256
    phase = micro.square_inclusion(n, side=128)
    mats = [(1.0, 0.3), (100.0, 0.3)]
    loc, green, sph, dev = _problem(phase, mats, 50.5, 0.3, variant)
    E = np.array([0., 0., 1.])
    checks = [1, 2, 5, 20, 100, 200]
    snaps = {}

    def cb(it, eps):
        if it + 1 in checks:
            snaps[it + 1] = eps.copy()
    eps_o, res_o, tau_o = O.basic_scheme(phase, sph, dev, 50.5, 0.3, E, 200, variant=variant,
                                         callback=cb)
    solver = BasicScheme(green, loc)
    solver.set_load(E)
    eps = solver.new_field()
    eps[...] = torch.from_numpy(E).cuda()
    done = 0
    for c in checks:
        for _ in range(c - done):
            solver.step(eps)
        done = c
        got = eps[0].cpu().numpy()
        ref = snaps[c]
        err = np.abs(got - ref).max() / np.abs(ref).max()
        assert err <= 1e-12, (c, err)
    r = solver.run(E, 200)  # fresh run for the residual history
    np.testing.assert_allclose(r.residuals[:, 0], res_o, rtol=1e-10)
    np.testing.assert_allclose(r.mean_tau[0], tau_o, rtol=1e-11, atol=1e-13)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
def test_spheres_3d_six_loads(variant):
    """Config 2 at reduced size: 32^3 random spheres, 6 load cases at once."""
    phase, _ = micro.random_spheres(32, radius=4, volume_fraction=0.3, seed=2)
    mats = [(1.0, 0.3), (100.0, 0.2)]
    loc, green, sph, dev = _problem(phase, mats, 50.5, 0.3, variant)
    E = np.eye(6)
    r = BasicScheme(green, loc, nload=6).run(E, 25)
    eps = r.eps.cpu().numpy()
    for l in range(6):
        eps_o, res_o, tau_o = O.basic_scheme(phase, sph, dev, 50.5, 0.3, E[l], 25,
                                             variant=variant)
        err = np.abs(eps[l] - eps_o).max() / np.abs(eps_o).max()
        assert err <= 1e-12, (l, err)
        np.testing.assert_allclose(r.residuals[:, l], res_o, rtol=1e-10)
        np.testing.assert_allclose(r.mean_tau[l], tau_o, rtol=1e-11, atol=1e-12)


@pytest.mark.gpu
def test_tolerance_stop_and_determinism():
    phase, _ = micro.random_spheres(24, radius=3, volume_fraction=0.2, seed=5)
    loc, green, _, _ = _problem(phase, [(1.0, 0.3), (10.0, 0.3)], 5.5, 0.3, "filtered")
    E = np.zeros(6)
    E[5] = 1.0
    s = BasicScheme(green, loc)
    r1 = s.run(E, 500, tol=1e-10)
    assert r1.iterations < 500 and r1.residuals[-1, 0] <= 1e-10 < r1.residuals[-2, 0]
    r2 = s.run(E, 500, tol=1e-10)
    assert r2.iterations == r1.iterations
    np.testing.assert_array_equal(r1.residuals, r2.residuals)
    np.testing.assert_array_equal(r1.eps.cpu().numpy(), r2.eps.cpu().numpy())
