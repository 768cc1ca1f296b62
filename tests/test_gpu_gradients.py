"""Stiffness fields and adjoint gradients on the GPU.

* the per-voxel field form of the local operator against the oracle;
* the strain / adjoint-strain contraction kernel against the oracle;
* dC_1212/dmu(x) by the adjoint autograd.Function against central
  differences (h = 1e-4 relative) of the GPU solver, on seeded voxels and
  seeded random directions, and against central differences of the oracle's
  CPU basic scheme;
* batching, the recompute checkpoint and the mixed-precision forward.
"""
import ctypes

import numpy as np
import pytest
import torch

from janus_b200 import _lib
from janus_b200 import microstructures as micro
from janus_b200.gradients import (StiffnessFieldProblem, effective_shear_modulus,
                                  mean_stress)
from janus_b200.operators import LocalPhaseOperator
from oracle import janus_oracle as O

dev = "cuda"


def _mu(n, dim, seed, std=1.0, corr=3.0):
    return np.exp(micro.gaussian_field(n, dim=dim, corr_len=corr, std=std, seed=seed))


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_field_local_operator_matches_oracle(dim):
    n = 24 if dim == 3 else 64
    shape = (n,) * dim
    s = 3 if dim == 2 else 6
    rng = np.random.default_rng(0)
    sph = rng.uniform(-2, 5, n ** dim)
    dv = rng.uniform(-1, 3, n ** dim)
    loc = LocalPhaseOperator(dim, shape, None, sph, dv)
    x = rng.standard_normal(shape + (s,))
    xd = torch.from_numpy(x).to(dev)
    y = torch.empty_like(xd)
    loc.apply_device(xd, y)
    ref = O.phase_apply(x, np.arange(n ** dim).reshape(shape), sph, dv, dim)
    assert np.array_equal(y.cpu().numpy(), ref)


@pytest.mark.gpu
def test_field_local_operator_rejects_wrong_size():
    with pytest.raises(ValueError):
        LocalPhaseOperator(2, (8, 8), None, np.ones(63), np.ones(63))


@pytest.mark.gpu
@pytest.mark.parametrize("dim,dtype", [(2, torch.float64), (3, torch.float64),
                                       (3, torch.float32)])
def test_local_gradient_kernel_matches_oracle(dim, dtype):
    n = 32 if dim == 3 else 96
    s = 3 if dim == 2 else 6
    L = 3
    rng = np.random.default_rng(1)
    e = rng.standard_normal((L,) + (n,) * dim + (s,))
    z = rng.standard_normal((L,) + (n,) * dim + (s,))
    ed = torch.from_numpy(e).to(dev, dtype)
    zd = torch.from_numpy(z).to(dev, dtype)
    nvox = n ** dim
    out = torch.empty((nvox, 2), dtype=torch.float64, device=dev)
    _lib.check(_lib.lib().jb_local_gradient(
        dim, 0 if dtype == torch.float64 else 1, nvox, L, ctypes.c_void_p(ed.data_ptr()),
        ctypes.c_void_p(zd.data_ptr()), 0.25, ctypes.c_void_p(out.data_ptr()), None))
    ref = O.local_gradient(ed.double().cpu().numpy(), zd.double().cpu().numpy(), dim, 0.25)
    np.testing.assert_allclose(out.cpu().numpy(), ref.reshape(nvox, 2), rtol=1e-12,
                               atol=1e-12)


def _c1212(mu, prob):
    with torch.no_grad():
        return float(effective_shear_modulus(mu, prob))


@pytest.mark.gpu
@pytest.mark.parametrize("mixed", [False, True])
def test_adjoint_gradient_matches_central_differences_3d(mixed):
    n = 16
    mu = torch.from_numpy(_mu(n, 3, seed=2)).to(dev)
    mu0 = 0.5 * float(mu.min() + mu.max())
    prob = StiffnessFieldProblem(nu=0.3, mu0=mu0, tol=1e-12, mixed=mixed, inner=20)
    m = mu.clone().requires_grad_(True)
    c = effective_shear_modulus(m, prob)
    c.backward()
    grad = m.grad.detach().cpu().numpy()
    scale = np.abs(grad).max()
    rng = np.random.default_rng(7)
    # 32 seeded voxels
    for v in rng.choice(n ** 3, 32, replace=False):
        idx = np.unravel_index(v, (n,) * 3)
        h = 1e-4 * float(mu[idx])
        vals = []
        for sgn in (1.0, -1.0):
            mp = mu.clone()
            mp[idx] += sgn * h
            vals.append(_c1212(mp, prob))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - grad[idx]) <= 2e-4 * scale, (idx, fd, grad[idx])
    # 4 seeded random directions
    for _ in range(4):
        d = torch.from_numpy(rng.standard_normal((n,) * 3)).to(dev)
        h = 1e-4
        vals = [_c1212(mu * (1 + sgn * h * d), prob) for sgn in (1.0, -1.0)]
        fd = (vals[0] - vals[1]) / (2 * h)
        an = float((m.grad * mu * d).sum())
        # the mean stress is linear in the solver's residual: each solve carries
        # ~tol of noise, which the difference divides by 2h (~1e-6 relative
        # here); the Krylov path varies between the perturbed solves, the FP64
        # basic scheme does not
        rtol = 1e-5 if mixed else 1e-6
        assert abs(fd - an) <= rtol * abs(an) + 1e-10, (fd, an)


@pytest.mark.gpu
def test_adjoint_gradient_matches_oracle_differences_2d():
    """GPU adjoint gradient against central differences of the oracle's
    CPU basic scheme on the same stiffness field."""
    n, nu = 16, 0.3
    mu_np = _mu(n, 2, seed=4, std=0.8, corr=2.0)
    g0 = 0.5 * (mu_np.min() + mu_np.max())
    E = np.array([0.0, 0.0, 1.0])
    prob = StiffnessFieldProblem(nu=nu, mu0=g0, tol=1e-14, mixed=False, max_iter=5000)
    m = torch.from_numpy(mu_np).to(dev).requires_grad_(True)
    effective_shear_modulus(m, prob).backward()
    grad = m.grad.cpu().numpy()
    rng = np.random.default_rng(3)
    for v in rng.choice(n * n, 4, replace=False):
        h = 1e-4 * mu_np.flat[v]
        vals = []
        for sgn in (1, -1):
            mp = mu_np.copy()
            mp.flat[v] += sgn * h
            vals.append(0.5 * O.field_mean_stress(mp, nu, g0, nu, E, 5000, 1e-14)[2])
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - grad.flat[v]) <= 1e-6 * np.abs(grad).max(), (v, fd, grad.flat[v])


@pytest.mark.gpu
def test_mean_stress_matches_oracle_forward():
    n, nu = 16, 0.3
    mu_np = _mu(n, 2, seed=6, std=0.8, corr=2.0)
    g0 = 0.5 * (mu_np.min() + mu_np.max())
    prob = StiffnessFieldProblem(nu=nu, mu0=g0, tol=1e-13, mixed=False, max_iter=5000)
    S = mean_stress(torch.from_numpy(mu_np).to(dev), prob).cpu().numpy()
    for j in range(3):
        E = np.eye(3)[j]
        ref = O.field_mean_stress(mu_np, nu, g0, nu, E, 5000, 1e-13)
        np.testing.assert_allclose(S[j], ref, rtol=1e-10, atol=1e-10 * np.abs(ref).max())


@pytest.mark.gpu
def test_batched_and_recomputed_gradients_agree():
    n = 12
    mus = torch.stack([torch.from_numpy(_mu(n, 3, seed=s)) for s in (10, 11)]).to(dev)
    base = dict(nu=0.3, tol=1e-11, mixed=True)
    mb = mus.clone().requires_grad_(True)
    cb = effective_shear_modulus(mb, StiffnessFieldProblem(**base), batched=True)
    assert cb.shape == (2,)
    cb.sum().backward()
    for b in range(2):
        m1 = mus[b].clone().requires_grad_(True)
        p = StiffnessFieldProblem(**base, keep_strain=False)
        c1 = effective_shear_modulus(m1, p)
        c1.backward()
        assert any(kind == "recompute" for kind, _, _ in p.stats)
        c1v, cbv = float(c1.detach()), float(cb.detach()[b])
        assert abs(c1v - cbv) <= 1e-12 * abs(c1v)
        g1, gb = m1.grad, mb.grad[b]
        assert float((g1 - gb).abs().max()) <= 1e-10 * float(g1.abs().max())


@pytest.mark.gpu
def test_full_mean_stress_gradient_uses_adjoint_rows():
    """A cotangent on every load case: the adjoint solve takes the nonzero
    cotangent rows as its macroscopic strains."""
    n = 12
    mu = torch.from_numpy(_mu(n, 3, seed=12)).to(dev)
    mu0 = 0.5 * float(mu.min() + mu.max())
    prob = StiffnessFieldProblem(nu=0.3, mu0=mu0, tol=1e-12, mixed=False)
    m = mu.clone().requires_grad_(True)
    S = mean_stress(m, prob)
    w = torch.zeros_like(S)
    w[0, 1] = 1.0
    w[3, 3] = -2.0
    (S * w).sum().backward()
    kinds = [k for k, _, _ in prob.stats]
    assert kinds == ["forward", "adjoint"]
    rng = np.random.default_rng(2)
    d = torch.from_numpy(rng.standard_normal((n,) * 3)).to(dev)
    h = 1e-4
    with torch.no_grad():
        p2 = StiffnessFieldProblem(nu=0.3, mu0=mu0, tol=1e-12, mixed=False)
        vals = [float((mean_stress(mu * (1 + s * h * d), p2) * w).sum()) for s in (1.0, -1.0)]
    fd = (vals[0] - vals[1]) / (2 * h)
    an = float((m.grad * mu * d).sum())
    assert abs(fd - an) <= 1e-6 * abs(an) + 1e-12, (fd, an)
