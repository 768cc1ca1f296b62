"""Row passes along 384-, 512-, 768- and 1024-point axes (the persistent long-row
kernels for three-component fields, the runtime-plan row kernels for the FFT
objects): the FFT objects against numpy's FFT with the reference's tolerance
model (tests/test_fft.py:9-80 of the reference), and the basic scheme on
grids whose rows are that long against the oracle, per iterate
(janus/fft/serial/_serial_fft.pyx:152-163 r2c, 177-190 c2r; the scheme of
sphinx/tutorials/square_basic/square_basic.py:83-97)."""
import numpy as np
import pytest
import torch

import janus_b200.material.elastic.linear.isotropic as material
from janus_b200 import operators as ops
from janus_b200.fft import serial
from janus_b200.green import filtered, truncated
from janus_b200.solvers import GMRES, BasicScheme, MixedScheme
from oracle import janus_oracle as O

# tile widths 2 and 3 (FP64 and FP32 solver rows), 2 (FFT objects), odd and
# ragged row counts
FFT_SHAPES = [(12, 1024), (5, 1024), (16, 512), (7, 512), (4, 8, 1024), (3, 6, 512)]


def _rel_l1(actual, expected):
    return np.sum(np.abs(actual - expected)) / np.sum(np.abs(expected))


@pytest.mark.gpu
@pytest.mark.parametrize("shape", FFT_SHAPES)
@pytest.mark.parametrize("dtype, delta", [(torch.float64, 1e-14), (torch.float32, 2e-6)])
def test_long_row_fft(shape, dtype, delta):
    transform = serial.create_real(shape, dtype=dtype)
    rng = np.random.default_rng(11)
    a = 2.0 * rng.random(transform.ishape) - 1.0
    out = np.asarray(transform.r2c(torch.from_numpy(a).to("cuda", dtype)).cpu(), dtype=np.float64)
    spec = out[..., 0::2] + 1j * out[..., 1::2]
    assert _rel_l1(spec, np.fft.rfftn(a)) <= delta
    back = transform.c2r(transform.r2c(torch.from_numpy(a).to("cuda", dtype)))
    assert _rel_l1(np.asarray(back.cpu(), dtype=np.float64), a) <= delta


def _problem(phase, g0, nu0, variant, dtype=None):
    mats = [(1.0, 0.3), (100.0, 0.2)]
    pars = [O.delta_c(g, nu, g0, nu0, 2) for g, nu in mats]
    tens = [ops.isotropic_4(s, d, 2) for s, d in pars]
    loc = ops.BlockDiagonalOperator2D.from_phases(phase, tens, dtype=dtype)
    fac = filtered if variant == "filtered" else truncated
    green = fac(material.create(g0, nu0, 2).green_operator(), phase.shape, 1.0, dtype=dtype)
    return loc, green, [p[0] for p in pars], [p[1] for p in pars]


def _phase(shape, seed):
    rng = np.random.default_rng(seed)
    return (rng.random(shape) < 0.3).astype(np.int32)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(32, 1024), (48, 512), (40, 768), (24, 384)])
@pytest.mark.parametrize("variant", ["filtered", "truncated"])
def test_long_rows_basic_scheme_per_iterate(shape, variant):
    """FP64: every iterate within 1e-12 of the oracle; FP32 (rows of width 3)
    within FP32 rounding of it."""
    phase = _phase(shape, 5)
    E = np.array([0.3, -0.1, 1.0])
    iters = 8
    eps_o, res_o, _ = O.basic_scheme(phase, *_problem(phase, 50.5, 0.3, variant)[2:], 50.5, 0.3,
                                     E, iters, variant=variant)
    for dtype, tol in ((torch.float64, 1e-12), (torch.float32, 2e-5)):
        loc, green, _, _ = _problem(phase, 50.5, 0.3, variant, dtype)
        r = BasicScheme(green, loc).run(E, iters)
        got = r.eps[0].double().cpu().numpy()
        err = np.abs(got - eps_o).max() / np.abs(eps_o).max()
        assert err <= tol, (dtype, err)
        if dtype == torch.float64:
            np.testing.assert_allclose(r.residuals[:, 0], res_o, rtol=1e-10)


@pytest.mark.gpu
def test_long_rows_mixed_scheme():
    """FP32 corrections (the residual epilogue of the long-row c2r pass) with
    FP64 defect correction converge to the FP64 solver's field."""
    phase = _phase((64, 1024), 7)
    loc, green, _, _ = _problem(phase, 50.5, 0.3, "filtered")
    E = np.eye(3)
    ref = BasicScheme(green, loc, nload=3).run(E, 3000, tol=1e-10)
    mix = MixedScheme(green, loc, nload=3, inner=10).run(E, tol=1e-10, max_outer=200)
    assert ref.converged and mix.converged
    err = (ref.eps - mix.eps).abs().max().item() / ref.eps.abs().max().item()
    assert err <= 1e-7, err


# Rows x load cases well above twice the persistent grid of the long-row
# kernels, so every CTA walks several rows through both buffers; ragged row
# counts, so the CTAs' row runs cross load cases at different points.
MANY_ROWS = [(512, 1024), (700, 512), (37, 1024), (300, 768), (1100, 384)]


def _per_load(phase, E, iters, variant, dtype, tol, loc_fn, oracle_fn):
    """BasicScheme with len(E) load cases against the oracle, per load case."""
    loc, green = loc_fn(dtype), _green(phase.shape, variant, dtype)
    r = BasicScheme(green, loc, nload=len(E)).run(E, iters)
    for l, El in enumerate(E):
        eps_o, res_o = oracle_fn(El)
        got = r.eps[l].double().cpu().numpy()
        err = np.abs(got - eps_o).max() / np.abs(eps_o).max()
        assert err <= tol, (dtype, l, err)
        if dtype == torch.float64:
            np.testing.assert_allclose(r.residuals[:, l], res_o, rtol=1e-10)


def _green(shape, variant, dtype):
    fac = filtered if variant == "filtered" else truncated
    return fac(material.create(50.5, 0.3, 2).green_operator(), shape, 1.0, dtype=dtype)


E3 = np.array([[1.0, 0.0, 0.0], [0.0, 1.0, 0.0], [0.3, -0.1, 1.0]])
TOLS = ((torch.float64, 1e-12), (torch.float32, 2e-5))


@pytest.mark.gpu
@pytest.mark.parametrize("shape", MANY_ROWS)
def test_many_long_rows_three_loads(shape):
    """Two phases (uint8 map), filtered, three load cases, per iterate."""
    phase = _phase(shape, 9)
    _, _, sph, dev = _problem(phase, 50.5, 0.3, "filtered")
    for dtype, tol in TOLS:
        _per_load(phase, E3, 4, "filtered", dtype, tol,
                  lambda dt: _problem(phase, 50.5, 0.3, "filtered", dt)[0],
                  lambda El: O.basic_scheme(phase, sph, dev, 50.5, 0.3, El, 4,
                                            variant="filtered")[:2])


@pytest.mark.gpu
def test_long_rows_int32_phase_map():
    """300 phases: the phase ids travel as int32 beside each row."""
    shape = (96, 1024)
    rng = np.random.default_rng(4)
    phase = rng.integers(0, 300, size=shape).astype(np.int32)
    mats = [(1.0 + 0.5 * p, 0.2 + 0.0005 * p) for p in range(300)]
    pars = [O.delta_c(g, nu, 50.5, 0.3, 2) for g, nu in mats]
    sph, dev = [p[0] for p in pars], [p[1] for p in pars]

    def loc(dt):
        return ops.BlockDiagonalOperator2D.from_phases(
            phase, [ops.isotropic_4(s, d, 2) for s, d in pars], dtype=dt)
    for dtype, tol in TOLS:
        _per_load(phase, E3[2:], 4, "truncated", dtype, tol, loc,
                  lambda El: O.basic_scheme(phase, sph, dev, 50.5, 0.3, El, 4,
                                            variant="truncated")[:2])


@pytest.mark.gpu
def test_long_rows_stiffness_field():
    """One (sph, dev) pair per voxel: the voxel index is the table entry."""
    shape = (64, 512)
    rng = np.random.default_rng(6)
    sph = rng.uniform(-20.0, 40.0, size=shape[0] * shape[1])
    dev = rng.uniform(-30.0, 60.0, size=shape[0] * shape[1])
    idx = np.arange(shape[0] * shape[1]).reshape(shape)
    for dtype, tol in TOLS:
        _per_load(idx, E3, 4, "filtered", dtype, tol,
                  lambda dt: ops.LocalPhaseOperator(2, shape, None, sph, dev, dtype=dt),
                  lambda El: O.basic_scheme(idx, sph, dev, 50.5, 0.3, El, 4,
                                            variant="filtered")[:2])


@pytest.mark.gpu
def test_long_rows_matrix_phases():
    """Full 3 x 3 matrices per phase (rotated cubic grains)."""
    shape = (80, 1024)
    phase = _phase(shape, 12)
    mats = np.stack([O.cubic2d_matrix(3.0, 1.0, 2.0, 0.3) - 50.5 * np.eye(3),
                     O.cubic2d_matrix(80.0, 30.0, 45.0, 1.1) - 50.5 * np.eye(3)])
    for dtype, tol in TOLS:
        _per_load(phase, E3[:1], 4, "truncated", dtype, tol,
                  lambda dt: ops.LocalPhaseOperator(2, shape, phase, None, None, dtype=dt,
                                                    matrices=mats),
                  lambda El: O.basic_scheme(phase, None, None, 50.5, 0.3, El, 4,
                                            variant="truncated", mats=mats)[:2])


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(300, 1024), (45, 512), (96, 768), (768, 768), (384, 384),
                                   (192, 384)])
@pytest.mark.parametrize("variant", ["filtered", "truncated"])
def test_long_rows_green_apply(shape, variant):
    """The plain r2c / c2r passes (no local operator, no epilogue) through
    the Green operator's apply, against the oracle."""
    rng = np.random.default_rng(21)
    x = rng.normal(size=shape + (3,))
    g = _green(shape, variant, torch.float64)
    y = np.asarray(g.apply(x))
    ref = O.green_apply(x, 50.5, 0.3, 1.0, variant)
    np.testing.assert_allclose(y, ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())


@pytest.mark.gpu
def test_many_long_rows_mixed_and_gmres():
    """The right-hand-side epilogue: FP32 mixed corrections and FP64 GMRES
    (d <- rhs - y) converge to the basic scheme's field on 512 x 1024 rows."""
    phase = _phase((512, 1024), 13)
    loc, green, _, _ = _problem(phase, 50.5, 0.3, "filtered")
    ref = BasicScheme(green, loc, nload=3).run(E3, 3000, tol=1e-10)
    mix = MixedScheme(green, loc, nload=3, inner=10).run(E3, tol=1e-10, max_outer=200)
    gm = GMRES(green, loc, nload=3).run(E3, tol=1e-10, max_iter=400)
    assert ref.converged and mix.converged and gm.converged
    for other in (mix, gm):
        err = (ref.eps - other.eps).abs().max().item() / ref.eps.abs().max().item()
        assert err <= 1e-7, err
