"""Row passes along 512- and 1024-point axes (one or two rows per CTA of the
runtime-plan row kernels): the FFT objects against numpy's FFT with the
reference's tolerance
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
from janus_b200.solvers import BasicScheme, MixedScheme
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
@pytest.mark.parametrize("shape", [(32, 1024), (48, 512)])
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
