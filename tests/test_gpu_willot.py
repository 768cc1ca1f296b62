"""The finite-difference (Willot 2015) discrete Green operator
(janus/green.pyx:976-1036): per-index matrices bitwise against the oracle
(itself pinned to the compiled reference), field-wide apply and the basic
scheme against the oracle, FP64 and FP32."""
import itertools

import numpy as np
import pytest
import torch

import janus_b200.material.elastic.linear.isotropic as material
from janus_b200 import operators as ops
from janus_b200.green import willot2015, FiniteDifferences2D, FiniteDifferences3D
from janus_b200.solvers import BasicScheme, MixedScheme
from oracle import janus_oracle as O


@pytest.mark.gpu
@pytest.mark.parametrize("n", [(8, 8), (6, 10), (4, 4, 4), (4, 6, 8)])
def test_willot_matrix_matches_oracle(n):
    dim = len(n)
    g = willot2015(material.create(0.75, 0.3, dim).green_operator(), n, 1.0)
    assert isinstance(g, FiniteDifferences2D if dim == 2 else FiniteDifferences3D)
    for b in itertools.product(*[range(v) for v in n]):
        g.set_frequency(np.asarray(b, dtype=np.intc))
        np.testing.assert_array_equal(np.asarray(g.to_memoryview()),
                                      O.willot_matrix(b, n, 1.0, 0.75, 0.3))


@pytest.mark.gpu
@pytest.mark.parametrize("shape,dtype", [((64, 48), torch.float64), ((32, 24, 20), torch.float64),
                                         ((128, 128), torch.float32),
                                         ((32, 32, 32), torch.float32),
                                         ((128, 128, 128), torch.float64)])
def test_willot_apply_matches_oracle(shape, dtype):
    dim = len(shape)
    s = 3 if dim == 2 else 6
    g = willot2015(material.create(0.75, 0.3, dim).green_operator(), shape, 1.0, dtype=dtype)
    rng = np.random.default_rng(1)
    x = rng.standard_normal(shape + (s,))
    y = g.apply(torch.from_numpy(x).to("cuda", dtype)).double().cpu().numpy()
    ref = O.green_apply(x.astype(np.float32).astype(np.float64) if dtype == torch.float32
                        else x, 0.75, 0.3, 1.0, "willot")
    tol = 1e-13 if dtype == torch.float64 else 2e-5
    assert np.abs(y - ref).max() <= tol * np.abs(ref).max()
    # in place
    xd = torch.from_numpy(x).to("cuda", dtype)
    g.apply(xd, xd)
    assert np.abs(xd.double().cpu().numpy() - y).max() <= tol * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(48, 40), (16, 20, 24)])
def test_willot_basic_scheme_matches_oracle(shape):
    dim = len(shape)
    rng = np.random.default_rng(4)
    phase = rng.integers(0, 2, size=shape).astype(np.uint8)
    g0, nu0 = 5.0, 0.3
    pars = [O.delta_c(1.0, 0.3, g0, nu0, dim), O.delta_c(10.0, 0.25, g0, nu0, dim)]
    tens = [ops.isotropic_4(a, b, dim) for a, b in pars]
    cls = ops.BlockDiagonalOperator2D if dim == 2 else ops.BlockDiagonalOperator3D
    loc = cls.from_phases(phase, tens)
    green = willot2015(material.create(g0, nu0, dim).green_operator(), shape, 1.0)
    s = dim * (dim + 1) // 2
    E = np.zeros(s)
    E[-1] = 1.0
    r = BasicScheme(green, loc, nload=1).run(E[None], 15)
    eps_o, res_o, tau_o = O.basic_scheme(phase, [p[0] for p in pars], [p[1] for p in pars],
                                         g0, nu0, E, 15, variant="willot")
    np.testing.assert_allclose(r.eps[0].cpu().numpy(), eps_o, rtol=1e-12, atol=1e-13)
    np.testing.assert_allclose(r.residuals[:, 0], res_o, rtol=1e-10)
    # the mixed solvers converge to the same FP64 solution (reference medium
    # inside the basic scheme's convergence range: mu0 > mu_max / 2)
    g0 = 6.0
    pars = [O.delta_c(1.0, 0.3, g0, nu0, dim), O.delta_c(10.0, 0.25, g0, nu0, dim)]
    loc = cls.from_phases(phase, [ops.isotropic_4(a, b, dim) for a, b in pars])
    green = willot2015(material.create(g0, nu0, dim).green_operator(), shape, 1.0)
    ref = BasicScheme(green, loc, nload=1).run(E[None], 5000, tol=1e-11)
    assert ref.residuals[-1].max() <= 1e-11
    for method in ("basic", "bicgstab"):
        m = MixedScheme(green, loc, nload=1, inner=20, method=method).run(E[None], tol=1e-11)
        assert m.residuals[-1].max() <= 1e-11
        err = (m.eps - ref.eps).abs().max().item() / ref.eps.abs().max().item()
        assert err <= 1e-8
