"""Restarted GMRES on the Lippmann-Schwinger equation, on the GPU, against
scipy's gmres over the oracle's operator x + Gamma0[(C - C0):x] (the
reference's Krylov route, examples/square_inclusion_scipy.py:52-59, 88), the
oracle's own residual of the returned fields, and the converged basic
scheme."""
import numpy as np
import pytest
import scipy.sparse.linalg as spla
import torch

import janus_b200.material.elastic.linear.isotropic as material
from janus_b200 import microstructures as micro
from janus_b200 import operators as ops
from janus_b200.green import filtered, truncated
from janus_b200.solvers import GMRES, BasicScheme, LippmannSchwingerOperator
from oracle import janus_oracle as O

FACTORY = {"truncated": truncated, "filtered": filtered}


def _problem(phase, mats, g0, nu0, variant, dtype=torch.float64):
    dim = phase.ndim
    pars = [O.delta_c(g, nu, g0, nu0, dim) for g, nu in mats]
    tens = [ops.isotropic_4(s, d, dim) for s, d in pars]
    cls = ops.BlockDiagonalOperator2D if dim == 2 else ops.BlockDiagonalOperator3D
    loc = cls.from_phases(phase, tens, dtype=dtype)
    green = FACTORY[variant](material.create(g0, nu0, dim).green_operator(), phase.shape, 1.0,
                             dtype=dtype)
    return loc, green, [p[0] for p in pars], [p[1] for p in pars]


def _oracle_op(phase, sph, dev, g0, nu0, variant):
    dim = phase.ndim
    s = 3 if dim == 2 else 6
    shape = phase.shape + (s,)
    G = O.spectral_green_field(phase.shape, 1.0, g0, nu0, variant)

    def mv(x):
        xx = x.reshape(shape)
        t = O.phase_apply(xx, phase, sph, dev, dim)
        return (xx + O.green_apply(t, g0, nu0, 1.0, variant, G=G)).ravel()
    n = int(np.prod(shape))
    return spla.LinearOperator((n, n), matvec=mv, dtype=np.float64), mv


def _oracle_residual(mv, eps, E):
    n = eps.size // E.size
    r = np.broadcast_to(E, eps.shape).ravel() - mv(eps.ravel())
    return np.linalg.norm(r) / (np.sqrt(n) * np.linalg.norm(E))


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
def test_gmres_2d_matches_scipy_on_the_oracle_operator(variant):
    phase = micro.square_inclusion(48, side=20)[:, :40].copy()
    mats, g0, nu0 = [(1.0, 0.3), (10.0, 0.25)], 5.5, 0.3
    loc, green, sph, dev = _problem(phase, mats, g0, nu0, variant)
    E = np.array([[0.0, 0.0, 1.0], [1.0, -0.5, 0.0]])
    res = GMRES(green, loc, nload=2, restart=20).run(E, tol=1e-12, max_iter=500)
    assert np.all(res.final_residuals <= 1e-12)
    aop, mv = _oracle_op(phase, sph, dev, g0, nu0, variant)
    eps = res.eps.cpu().numpy()
    for l in range(2):
        b = np.broadcast_to(E[l], phase.shape + (3,)).ravel().copy()
        x, info = spla.gmres(aop, b, rtol=1e-13, atol=0.0, restart=20, maxiter=200)
        assert info == 0
        assert np.abs(eps[l].ravel() - x).max() <= 1e-9 * np.abs(x).max()
        # the oracle's own residual of the GPU solution
        r = _oracle_residual(mv, eps[l], E[l])
        assert r <= 2e-12 and abs(r - res.final_residuals[l]) <= 1e-13


@pytest.mark.gpu
def test_gmres_3d_six_loads_filtered():
    phase, _ = micro.random_spheres(16, radius=3, volume_fraction=0.25, seed=4)
    mats, g0, nu0 = [(1.0, 0.3), (100.0, 0.2)], 50.5, 0.3
    loc, green, sph, dev = _problem(phase, mats, g0, nu0, "filtered")
    E = np.eye(6)
    res = GMRES(green, loc, nload=6, restart=30).run(E, tol=1e-10, max_iter=2000)
    assert np.all(res.final_residuals <= 1e-10)
    _, mv = _oracle_op(phase, sph, dev, g0, nu0, "filtered")
    eps = res.eps.cpu().numpy()
    for l in range(6):
        assert _oracle_residual(mv, eps[l], E[l]) <= 2e-10
    # mean (C - C0):eps against the oracle's tables on the same field
    tau = np.stack([O.phase_apply(eps[l], phase, sph, dev, 3).mean(axis=(0, 1, 2))
                    for l in range(6)])
    np.testing.assert_allclose(res.mean_tau, tau, rtol=1e-12, atol=1e-12)


@pytest.mark.gpu
def test_gmres_agrees_with_the_converged_basic_scheme_and_needs_fewer_iterations():
    phase = micro.square_inclusion(64, side=32)
    mats, g0, nu0 = [(1.0, 0.3), (100.0, 0.3)], 50.5, 0.3
    loc, green, _, _ = _problem(phase, mats, g0, nu0, "truncated")
    E = np.array([0.0, 0.0, 1.0])
    gm = GMRES(green, loc, restart=30).run(E, tol=1e-11, max_iter=1000)
    bs = BasicScheme(green, loc).run(E, 20000, tol=1e-13)
    assert gm.final_residuals[0] <= 1e-11 and bs.residuals[-1, 0] <= 1e-13
    d = (gm.eps - bs.eps).abs().max().item()
    assert d <= 1e-8 * bs.eps.abs().max().item()
    assert gm.iterations * 5 < bs.iterations


@pytest.mark.gpu
def test_gmres_restarts_history_and_initial_guess():
    phase = micro.square_inclusion(32, side=12)
    loc, green, _, _ = _problem(phase, [(1.0, 0.3), (30.0, 0.3)], 15.5, 0.3, "filtered")
    E = np.array([0.3, 0.0, 1.0])
    solver = GMRES(green, loc, restart=4)
    r = solver.run(E, tol=1e-10, max_iter=400)
    assert r.final_residuals[0] <= 1e-10 and r.iterations > 4
    h = r.residuals[:, 0]
    for c in range(0, len(h), 4):   # Givens estimates never grow within a cycle
        cyc = h[c:c + 4]
        assert np.all(np.diff(cyc) <= 1e-15 + 1e-12 * cyc[:-1])
    # a converged field is returned unchanged, with no Arnoldi step
    eps = r.eps.clone()
    r2 = solver.run(E, tol=1e-9, max_iter=100, eps=eps)
    assert r2.iterations == 0 and torch.equal(eps, r.eps)
    # max_iter bounds the work; the true residual is still reported
    r3 = solver.run(E, tol=1e-14, max_iter=3)
    assert r3.iterations == 3 and r3.final_residuals[0] > 1e-14


@pytest.mark.gpu
def test_scipy_gmres_over_the_gpu_operator():
    phase = micro.square_inclusion(32, side=16)
    mats, g0, nu0 = [(1.0, 0.3), (10.0, 0.3)], 5.5, 0.3
    loc, green, sph, dev = _problem(phase, mats, g0, nu0, "truncated")
    op = LippmannSchwingerOperator(green, loc)
    aop, mv = _oracle_op(phase, sph, dev, g0, nu0, "truncated")
    rng = np.random.default_rng(0)
    x = rng.standard_normal(op.shape[1])
    np.testing.assert_allclose(op.matvec(x), mv(x), rtol=1e-12, atol=1e-12)
    b = np.broadcast_to([0.0, 0.0, 1.0], (32, 32, 3)).ravel().copy()
    xs, info = spla.gmres(spla.aslinearoperator(op), b, rtol=1e-12, atol=0.0, restart=20)
    assert info == 0
    gm = GMRES(green, loc).run(np.array([0.0, 0.0, 1.0]), tol=1e-12)
    np.testing.assert_allclose(gm.eps.cpu().numpy().ravel(), xs, rtol=0, atol=1e-9)
    # rmatvec is the transpose: <A x, y> = <x, A^T y>
    y = rng.standard_normal(op.shape[0])
    assert abs(op.matvec(x) @ y - x @ op.rmatvec(y)) <= 1e-10 * abs(op.matvec(x) @ y)


@pytest.mark.gpu
def test_gmres_validation():
    phase = micro.square_inclusion(16, side=8)
    loc, green, _, _ = _problem(phase, [(1.0, 0.3), (2.0, 0.3)], 1.5, 0.3, "truncated")
    with pytest.raises(ValueError):
        GMRES(green, loc, restart=0)
    loc32, green32, _, _ = _problem(phase, [(1.0, 0.3), (2.0, 0.3)], 1.5, 0.3, "truncated",
                                    torch.float32)
    with pytest.raises(ValueError):
        GMRES(green32, loc32)
    with pytest.raises(ValueError):
        GMRES(green, loc).run(np.zeros(3))
