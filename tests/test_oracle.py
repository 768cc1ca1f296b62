"""Pins the oracle (oracle/janus_oracle.py) before it is trusted.

* against the reference's 18 golden Green-operator files (sampled fixture,
  tests/golden), with the reference's tolerance rtol=ULP, atol=10 ULP
  (tests/test_discrete_green_operator.py:199 of the reference);
* against the closed-form Green tensor of tests/test_greenop.py:21-35;
* against the published C_1212 of the square tutorial
  (sphinx/tutorials/square_basic/square_basic.rst:227);
* against the reference's own Cython path compiled with the FFT shim
  (oracle/_ref), when built.
"""
import itertools
import math

import numpy as np
import pytest

from oracle import janus_oracle as O
from tests.conftest import ULP, golden_cases, reference_checker
from tests.golden.make_golden import checksum_weights, unit_block


def test_oracle_matches_golden_files(golden):
    for key, variant, shape, comp, block, offs in golden_cases(golden):
        x = unit_block(shape, comp, block, offs)
        y = O.green_apply(x, 0.75, 0.3, 1.0, variant)
        idx = golden[key + "/idx"]
        ys = golden[key + "/y"]
        act = y.reshape(-1, y.shape[-1])[idx]
        np.testing.assert_allclose(act, ys, rtol=ULP, atol=10 * ULP, err_msg=key)
        cs = golden[key + "/checksums"]
        w = checksum_weights(shape, y.shape[-1])
        got = np.array([y.sum(), (y * y).sum(), (w * y).sum()])
        np.testing.assert_allclose(got, cs, rtol=1e-12, atol=1e-12, err_msg=key)


def _closed_form(k, g, nu, dim):
    # tests/test_greenop.py:21-35 of the reference, restated
    k = np.asarray(k, dtype=float)
    sym = dim * (dim + 1) // 2
    if np.sum(k * k) == 0:
        return np.zeros((sym, sym))
    n = k / np.sqrt(np.sum(k * k))
    if dim == 2:
        pairs = [(0, 0), (1, 1), (0, 1)]
    else:
        pairs = [(0, 0), (1, 1), (2, 2), (1, 2), (2, 0), (0, 1)]
    d = np.eye(dim)
    out = np.zeros((sym, sym))
    for a, (i, j) in enumerate(pairs):
        for b, (kk, ll) in enumerate(pairs):
            v = ((d[i, kk] * n[j] * n[ll] + d[i, ll] * n[j] * n[kk] + d[j, kk] * n[i] * n[ll]
                  + d[j, ll] * n[i] * n[kk]) - 2 * n[i] * n[j] * n[kk] * n[ll] / (1. - nu)) / (4 * g)
            fa = math.sqrt(2) if i != j else 1.0
            fb = math.sqrt(2) if kk != ll else 1.0
            out[a, b] = fa * fb * v
    return out


@pytest.mark.parametrize("dim", [2, 3])
def test_oracle_green_matrix_closed_form(dim):
    rng = np.random.default_rng(1)
    for _ in range(50):
        k = rng.normal(size=dim) * 3
        np.testing.assert_allclose(O.green_matrix(k, 0.7, 0.3), _closed_form(k, 0.7, 0.3, dim),
                                   rtol=1e-13, atol=1e-15)
    assert not O.green_matrix(np.zeros(dim), 0.7, 0.3).any()


def test_oracle_tutorial_known_answer():
    # square_basic.py:60-97: 256^2, corner square a = 1/2, mu_i=100/nu_i=0.2,
    # mu_m=1/nu_m=0.3, mu_0=50/nu_0=0.3, E=(0,0,1), 400 iterations
    dim, n = 2, 256
    phase = np.zeros((n, n), dtype=np.uint8)
    imax = int(np.ceil(n * 0.5 - 0.5))
    phase[:imax, :imax] = 1
    sm, dm = O.delta_c(1.0, 0.3, 50.0, 0.3, dim)
    si, di = O.delta_c(100.0, 0.2, 50.0, 0.3, dim)
    E = np.array([0., 0., 1.])
    eps, res, mean_tau = O.basic_scheme(phase, [sm, si], [dm, di], 50.0, 0.3, E, 400)
    c1212 = 50.0 + 0.5 * mean_tau[-1] / E[-1]
    assert abs(c1212 - 1.41903971282) < 5e-12
    assert res[-1] < res[0]


GRID_SIZES = [(8, 8), (8, 16), (16, 8), (4, 4, 4), (4, 8, 16), (16, 8, 4)]


_REF_FACTORY = {"truncated": "truncated", "filtered": "filtered", "willot": "willot2015"}
_ORACLE_MATRIX = {"truncated": O.truncated_matrix, "filtered": O.filtered_matrix,
                  "willot": O.willot_matrix}


@pytest.mark.parametrize("n", GRID_SIZES)
@pytest.mark.parametrize("variant", ["truncated", "filtered", "willot"])
def test_oracle_matrices_match_reference_build(n, variant):
    ref = reference_checker()
    if ref is None:
        pytest.skip("reference checker (oracle/_ref) not built")
    import janus.green as rgreen
    import janus.material.elastic.linear.isotropic as rmat
    dim = len(n)
    g = rmat.create(0.75, 0.3, dim).green_operator()
    op = getattr(rgreen, _REF_FACTORY[variant])(g, n, 1.0)
    mat = _ORACLE_MATRIX[variant]
    for b in itertools.product(*[range(v) for v in n]):
        op.set_frequency(np.asarray(b, dtype=np.intc))
        np.testing.assert_array_equal(np.asarray(op.to_memoryview()),
                                      mat(b, n, 1.0, 0.75, 0.3))


@pytest.mark.parametrize("variant", ["truncated", "filtered", "willot"])
@pytest.mark.parametrize("shape", [(12, 10), (6, 5, 8)])
def test_oracle_basic_scheme_matches_reference_build(variant, shape):
    ref = reference_checker()
    if ref is None:
        pytest.skip("reference checker (oracle/_ref) not built")
    import janus.fft.serial as rfft
    import janus.green as rgreen
    import janus.material.elastic.linear.isotropic as rmat
    import janus.operators as rops
    dim = len(shape)
    rng = np.random.default_rng(5)
    phase = rng.integers(0, 2, size=shape).astype(np.uint8)
    g0, nu0 = 5.0, 0.3
    pars = [O.delta_c(1.0, 0.3, g0, nu0, dim), O.delta_c(10.0, 0.25, g0, nu0, dim)]
    sph = [p[0] for p in pars]
    dev = [p[1] for p in pars]
    s = dim * (dim + 1) // 2
    E = np.zeros(s)
    E[-1] = 1.0
    iters = 12
    eps_o, res_o, tau_o = O.basic_scheme(phase, sph, dev, g0, nu0, E, iters, variant=variant)
    # the tutorial loop on the reference's own objects
    ops = np.empty(shape, dtype=object)
    tens = [rops.isotropic_4(a, b, dim) for a, b in zip(sph, dev)]
    for idx in np.ndindex(*shape):
        ops[idx] = tens[phase[idx]]
    loc = rops.block_diagonal_operator(ops)
    gr = getattr(rgreen, _REF_FACTORY[variant])(
        rmat.create(g0, nu0, dim).green_operator(), shape, 1.0, rfft.create_real(shape))
    eps = np.empty(shape + (s,))
    eps[...] = E
    new = np.empty_like(eps)
    norm = 1 / np.sqrt(np.prod(shape)) / np.linalg.norm(E)
    res = []
    for _ in range(iters):
        loc.apply(eps, new)
        gr.apply(new, new)
        np.subtract(E, new, out=new)
        res.append(norm * np.linalg.norm(new - eps))
        eps, new = new, eps
    np.testing.assert_allclose(eps_o, eps, rtol=1e-12, atol=1e-14)
    np.testing.assert_allclose(res_o, res, rtol=1e-10)


def _field_2d(n, seed, std=0.6):
    rng = np.random.default_rng(seed)
    g = rng.standard_normal((n, n))
    # smooth a little so that neighbouring voxels correlate
    g = 0.5 * g + 0.125 * (np.roll(g, 1, 0) + np.roll(g, -1, 0) + np.roll(g, 1, 1) +
                           np.roll(g, -1, 1))
    g = (g - g.mean()) * (std / g.std())
    return np.exp(g)


@pytest.mark.parametrize("cot", [(0.0, 0.0, 1.0), (0.3, -0.2, 1.0)])
def test_oracle_adjoint_gradient_matches_differences(cot):
    """The adjoint formula dJ/dmu(x) = (1/N) zeta.dC/dmu.eps, with zeta the
    basic-scheme solution for the cotangent as macroscopic strain, against
    central differences of the oracle's basic scheme (stiffness field, 2D)."""
    n, nu = 12, 0.3
    mu = _field_2d(n, 5)
    g0 = 0.5 * (mu.min() + mu.max())
    E = np.array([0.0, 0.0, 1.0])
    G = np.asarray(cot)
    tol, its = 1e-15, 3000
    phase, sph, dev = O.field_tables(mu, nu, g0, nu)
    eps, _, _ = O.basic_scheme(phase, sph, dev, g0, nu, E, its, tol=tol)
    zeta, _, _ = O.basic_scheme(phase, sph, dev, g0, nu, G, its, tol=tol)
    out = O.local_gradient(eps[None], zeta[None], 2, 1.0 / mu.size)
    grad = out[..., 0] * 2 * O.bulk_modulus(1.0, nu, 2) + out[..., 1] * 2.0
    rng = np.random.default_rng(1)
    for v in rng.choice(mu.size, 4, replace=False):
        h = 1e-4 * mu.flat[v]
        vals = []
        for sgn in (1, -1):
            m = mu.copy()
            m.flat[v] += sgn * h
            vals.append(G @ O.field_mean_stress(m, nu, g0, nu, E, its, tol))
        fd = (vals[0] - vals[1]) / (2 * h)
        assert abs(fd - grad.flat[v]) <= 1e-6 * abs(grad).max(), (v, fd, grad.flat[v])


@pytest.mark.parametrize("theta", [0.0, 0.3, 1.1, -2.0])
def test_oracle_cubic_tensor_matches_reference_build(theta):
    ref = reference_checker()
    if ref is None:
        pytest.skip("reference checker (oracle/_ref) not built")
    import janus.operators as rops
    t = rops.FourthRankCubicTensor2D(3.0, 1.2, 0.7, theta)
    np.testing.assert_array_equal(np.asarray(t.to_memoryview()),
                                  O.cubic2d_matrix(3.0, 1.2, 0.7, theta))


@pytest.mark.parametrize("theta", [0.0, 0.7])
def test_host_linear_and_cubic_operators_match_reference_build(theta):
    """janus_b200.operators.LinearOperator / FourthRankCubicTensor2D (host
    apply, to_memoryview) against the reference's compiled classes, bitwise."""
    ref = reference_checker()
    if ref is None:
        pytest.skip("reference checker (oracle/_ref) not built")
    import janus.operators as rops
    from janus_b200 import operators as mops
    rng = np.random.default_rng(2)
    x = rng.standard_normal(3)
    a = rng.standard_normal((3, 3))
    r_cub, m_cub = rops.FourthRankCubicTensor2D(3.0, 1.2, 0.7, theta), \
        mops.FourthRankCubicTensor2D(3.0, 1.2, 0.7, theta)
    np.testing.assert_array_equal(np.asarray(r_cub.apply(x)), m_cub.apply(x))
    np.testing.assert_array_equal(np.asarray(r_cub.to_memoryview()), m_cub.to_memoryview())
    r_lin, m_lin = rops.LinearOperator(a), mops.LinearOperator(a)
    np.testing.assert_array_equal(np.asarray(r_lin.apply(x)), m_lin.apply(x))
    np.testing.assert_array_equal(np.asarray(r_lin.apply_transpose(x)), m_lin.apply_transpose(x))
    np.testing.assert_array_equal(np.asarray(r_lin.to_memoryview()), m_lin.to_memoryview())
