"""Anisotropic local operators (LinearOperator, FourthRankCubicTensor2D:
janus/operators.pyx:195-254, 411-450) as phase tables of matrices: the
block-diagonal apply bitwise against the oracle, and the basic, mixed and
Krylov solvers on a 2D polycrystal of rotated cubic grains against the
oracle and the FP64 solver."""
import numpy as np
import pytest
import torch

import janus_b200.material.elastic.linear.isotropic as material
from janus_b200 import operators as ops
from janus_b200.green import filtered, truncated
from janus_b200.solvers import BasicScheme, MixedScheme
from oracle import janus_oracle as O


def _grains(n, count, seed):
    rng = np.random.default_rng(seed)
    sites = rng.uniform(0, n, size=(count, 2))
    i0, i1 = np.meshgrid(np.arange(n) + 0.5, np.arange(n) + 0.5, indexing="ij")
    d = np.full((n, n), np.inf)
    gid = np.zeros((n, n), dtype=np.int64)
    for k, (a, b) in enumerate(sites):
        d0 = np.abs(i0 - a)
        d1 = np.abs(i1 - b)
        dk = np.minimum(d0, n - d0) ** 2 + np.minimum(d1, n - d1) ** 2
        closer = dk < d
        d[closer] = dk[closer]
        gid[closer] = k
    return gid, rng.uniform(0, np.pi, size=count)


def _polycrystal(n=64, count=12, seed=0):
    gid, thetas = _grains(n, count, seed)
    mu0, k0 = 1.0, 2.2
    nu0 = (k0 - mu0) / (2 * k0)
    C0 = ops.isotropic_4(2 * k0, 2 * mu0, 2).to_memoryview()
    tens = []
    for th in thetas:
        c = ops.FourthRankCubicTensor2D(3.0, 1.2, 0.7, th)
        dC = c.to_memoryview() - C0
        tens.append(ops.LinearOperator(dC))
    return gid, tens, mu0, nu0


@pytest.mark.gpu
def test_block_diagonal_matrix_apply_bitwise():
    gid, tens, mu0, nu0 = _polycrystal(48, 9, 1)
    loc_obj = np.empty(gid.shape, dtype=object)
    for idx in np.ndindex(*gid.shape):
        loc_obj[idx] = tens[gid[idx]]
    bd = ops.BlockDiagonalOperator2D(loc_obj)
    assert bd.local is not None and bd.local.matrices is not None
    rng = np.random.default_rng(0)
    x = rng.standard_normal(gid.shape + (3,))
    mats = np.stack([t.to_memoryview() for t in tens])
    ref = O.block_linear_apply(mats[gid], x)
    assert np.array_equal(bd.apply(x), ref)
    fp = ops.BlockDiagonalOperator2D.from_phases(gid, tens)
    assert np.array_equal(fp.apply(x), ref)


@pytest.mark.gpu
def test_matrix_field_3d_apply_bitwise():
    n = 12
    rng = np.random.default_rng(3)
    mats = rng.standard_normal((n ** 3, 6, 6))
    loc = ops.LocalPhaseOperator(3, (n, n, n), None, None, None, matrices=mats)
    x = rng.standard_normal((n, n, n, 6))
    xd = torch.from_numpy(x).cuda()
    y = torch.empty_like(xd)
    loc.apply_device(xd, y)
    ref = O.block_linear_apply(mats.reshape(n, n, n, 6, 6), x)
    assert np.array_equal(y.cpu().numpy(), ref)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
def test_polycrystal_basic_scheme_matches_oracle(variant):
    gid, tens, mu0, nu0 = _polycrystal(64, 12, 2)
    loc = ops.BlockDiagonalOperator2D.from_phases(gid, tens)
    f = truncated if variant == "truncated" else filtered
    green = f(material.create(mu0, nu0, 2).green_operator(), gid.shape, 1.0)
    E = np.array([0.0, 0.0, 1.0])
    r = BasicScheme(green, loc, nload=1).run(E[None], 12)
    mats = np.stack([t.to_memoryview() for t in tens])
    eps_o, res_o, tau_o = O.basic_scheme(gid, None, None, mu0, nu0, E, 12, variant=variant,
                                         mats=mats)
    np.testing.assert_allclose(r.eps[0].cpu().numpy(), eps_o, rtol=1e-12, atol=1e-13)
    # the residual falls to ~1e-8; FP64 rounding of eps is ~1e-17 absolute
    np.testing.assert_allclose(r.residuals[:, 0], res_o, rtol=1e-10, atol=1e-15)
    np.testing.assert_allclose(r.mean_tau[0], tau_o, rtol=1e-11, atol=1e-13)


@pytest.mark.gpu
def test_polycrystal_mixed_solvers_match_fp64():
    gid, tens, mu0, nu0 = _polycrystal(128, 30, 4)
    loc = ops.BlockDiagonalOperator2D.from_phases(gid, tens)
    green = truncated(material.create(mu0, nu0, 2).green_operator(), gid.shape, 1.0)
    E = np.eye(3)
    ref = BasicScheme(green, loc, nload=3).run(E, 20000, tol=1e-11)
    assert ref.residuals[-1].max() <= 1e-11
    for method in ("basic", "bicgstab"):
        m = MixedScheme(green, loc, nload=3, inner=20, method=method).run(E, tol=1e-11)
        assert m.residuals[-1].max() <= 1e-11
        assert np.abs(m.mean_tau - ref.mean_tau).max() <= 1e-8 * np.abs(ref.mean_tau).max()
