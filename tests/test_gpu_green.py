"""Discrete Green operators on the GPU: golden files, oracle parity, the
per-frequency API and the reference's invalid-argument cases
(tests/test_discrete_green_operator.py of the reference)."""
import itertools

import numpy as np
import pytest
import torch

import janus_b200.fft.serial as fft
import janus_b200.material.elastic.linear.isotropic as material
from janus_b200.green import filtered, truncated
from oracle import janus_oracle as O
from tests.conftest import ULP, golden_cases
from tests.golden.make_golden import checksum_weights, unit_block

MU = 0.75
NU = 0.3
GRID_SIZES = ([(8, 8), (8, 16), (16, 8), (4, 4, 4)] + list(itertools.permutations((4, 8, 16))))
FACTORY = {"truncated": truncated, "filtered": filtered}


def multi_indices(n):
    return [np.asarray(b, dtype=np.intc) for b in itertools.product(*[range(v) for v in n])]


@pytest.mark.gpu
@pytest.mark.parametrize("flag", [0, 1, 2])
def test_apply_golden(golden, flag):
    """The 18 reference golden files, rtol=ULP, atol=10 ULP, with the three
    call forms apply(x), apply(x, x), apply(x, y)."""
    for key, variant, shape, comp, block, offs in golden_cases(golden):
        x = unit_block(shape, comp, block, offs)
        transform = fft.create_real(shape)
        green = FACTORY[variant](material.create(MU, NU, len(shape)).green_operator(), shape,
                                 1., transform=transform)
        if flag == 0:
            actual = green.apply(x)
        elif flag == 1:
            actual = green.apply(x, x)
        else:
            base = np.zeros(transform.ishape + (green.oshape[-1],), np.float64)
            actual = green.apply(x, base)
            assert actual.base is base
        actual = np.asarray(actual)
        idx = golden[key + "/idx"]
        np.testing.assert_allclose(actual.reshape(-1, actual.shape[-1])[idx], golden[key + "/y"],
                                   rtol=ULP, atol=10 * ULP, err_msg=key)
        w = checksum_weights(shape, actual.shape[-1])
        got = np.array([actual.sum(), (actual * actual).sum(), (w * actual).sum()])
        np.testing.assert_allclose(got, golden[key + "/checksums"], rtol=1e-12, atol=1e-12)
        # the whole field against the oracle
        np.testing.assert_allclose(actual, O.green_apply(unit_block(shape, comp, block, offs),
                                                         MU, NU, 1.0, variant),
                                   rtol=ULP, atol=10 * ULP, err_msg=key)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
@pytest.mark.parametrize("shape", [(64, 64), (31, 45), (16, 12, 10), (9, 7, 5), (1, 8),
                                   (24, 1, 6)])
def test_apply_random_fields_vs_oracle(variant, shape):
    rng = np.random.default_rng(11)
    s = 3 if len(shape) == 2 else 6
    x = rng.normal(size=shape + (s,))
    g = FACTORY[variant](material.create(MU, NU, len(shape)).green_operator(), shape, 0.5)
    y = np.asarray(g.apply(x))
    ref = O.green_apply(x, MU, NU, 0.5, variant)
    np.testing.assert_allclose(y, ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
    # torch in, torch out, in place
    xt = torch.from_numpy(x).cuda()
    out = g.apply(xt, xt)
    assert out is xt
    np.testing.assert_allclose(xt.cpu().numpy(), y, rtol=0, atol=0)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
@pytest.mark.parametrize("n", GRID_SIZES)
def test_to_memoryview(variant, n):
    dim = len(n)
    greenc = material.create(MU, NU, dim).green_operator()
    greend = FACTORY[variant](greenc, n, 1.0)
    mat = O.truncated_matrix if variant == "truncated" else O.filtered_matrix
    for b in multi_indices(n):
        greend.set_frequency(b)
        expected = mat(b, n, 1.0, MU, NU)
        actual = greend.to_memoryview()
        np.testing.assert_allclose(actual, expected, ULP, ULP)
        base = np.empty_like(expected)
        assert greend.to_memoryview(base).base is base


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
@pytest.mark.parametrize("n", GRID_SIZES)
def test_apply_by_freq_host_and_device(variant, n):
    dim = len(n)
    x = [np.array([0.3, -0.4, 0.5]), np.array([0.1, -0.2, 0.3, -0.4, 0.5, -0.6])][dim - 2]
    green = FACTORY[variant](material.create(MU, NU, dim).green_operator(), n, 1.)
    bs = multi_indices(n)
    expected = []
    for flag, b in zip(itertools.cycle(range(3)), bs):
        green.set_frequency(b)
        g = np.asarray(green.to_memoryview())
        exp = np.dot(g, x)
        expected.append(exp)
        base = None if flag == 0 else (x.copy() if flag == 1 else np.empty_like(exp))
        actual = green.apply_by_freq(x if flag != 1 else base, base)
        if flag != 0:
            assert actual.base is base
        np.testing.assert_allclose(actual, exp, ULP, ULP)
    # the device contraction used by apply(), on the same indices
    rng = np.random.default_rng(4)
    tau = rng.normal(size=(len(bs), x.size, 2))
    eta = green.apply_by_freq_device(np.stack(bs), tau).cpu().numpy()
    for i, b in enumerate(bs):
        green.set_frequency(b)
        g = np.asarray(green.to_memoryview())
        for part in range(2):
            ref = g @ tau[i, :, part]
            np.testing.assert_allclose(eta[i, :, part], ref, rtol=1e-14,
                                       atol=1e-14 * (np.abs(g).max() * np.abs(tau[i]).max()))


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
def test_init_invalid_params(variant):
    g2 = material.create(MU, NU, 2).green_operator()
    g3 = material.create(MU, NU, 3).green_operator()
    params = [(g3, (9, 9), 1., None), (g2, (-1, 9), 1., None), (g2, (9, -1), 1., None),
              (g2, (9, 9), -1., None), (g2, (9, 9), 1., fft.create_real((8, 9))),
              (g2, (9, 9), 1., fft.create_real((9, 8))), (g2, (9, 9, 9), 1., None),
              (g3, (-1, 9, 9), 1., None), (g3, (9, -1, 9), 1., None), (g3, (9, 9, -1), 1., None),
              (g3, (9, 9, 9), -1., None)]
    for greenc, n, h, transform in params:
        with pytest.raises(ValueError):
            FACTORY[variant](greenc, n, h, transform)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
def test_invalid_shapes(variant):
    g2 = FACTORY[variant](material.create(MU, NU, 2).green_operator(), (8, 16), 1.0)
    g3 = FACTORY[variant](material.create(MU, NU, 3).green_operator(), (8, 16, 32), 1.0)
    for g in (g2, g3):
        with pytest.raises(ValueError):
            g.to_memoryview(np.zeros((g.oshape[-1], g.ishape[-1] + 1)))
        with pytest.raises(ValueError):
            g.to_memoryview(np.zeros((g.oshape[-1] + 1, g.ishape[-1])))
        g.set_frequency(np.zeros(g.dim, dtype=np.intc))
        with pytest.raises(ValueError):
            g.apply_by_freq(np.zeros(g.ishape[-1]), np.zeros(g.oshape[-1] + 1))
        with pytest.raises(ValueError):
            g.apply_by_freq(np.zeros(g.ishape[-1] + 1), np.zeros(g.oshape[-1]))
        for i in range(len(g.ishape)):
            xs = list(g.ishape)
            xs[i] += 1
            with pytest.raises(ValueError):
                g.apply(np.zeros(xs), np.zeros(g.oshape))
            ys = list(g.oshape)
            ys[i] += 1
            with pytest.raises(ValueError):
                g.apply(np.zeros(g.ishape), np.zeros(ys))
        bad = np.array(g.ishape[:-1], dtype=np.intc)
        with pytest.raises(ValueError):
            g.set_frequency(bad)
        with pytest.raises(ValueError):
            g.set_frequency(np.zeros(g.dim + 1, dtype=np.intc))


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
@pytest.mark.parametrize("shape", [(64, 64), (31, 45), (48, 62), (1, 8), (128, 96),
                                   (256, 256), (9, 7, 5), (32, 24, 16)])
def test_apply_random_fields_fp32_vs_oracle(variant, shape):
    """FP32 apply, including 2D grids whose half-spectrum rows of m * 3
    complex floats are padded to 16 bytes inside the solver passes (m odd:
    64, 45, 96, 256; m even: 62), against the FP64 oracle."""
    rng = np.random.default_rng(12)
    s = 3 if len(shape) == 2 else 6
    x = rng.normal(size=shape + (s,))
    g = FACTORY[variant](material.create(MU, NU, len(shape)).green_operator(), shape, 0.5,
                         dtype="float32")
    y = g.apply(torch.from_numpy(x).float().cuda()).double().cpu().numpy()
    ref = O.green_apply(x, MU, NU, 0.5, variant)
    assert np.abs(y - ref).max() <= 2e-6 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(64, 64), (45, 31), (96, 62)])
def test_fp32_2d_basic_scheme_vs_oracle(shape):
    """The FP32 2D solver passes (local operator in the first, update and
    residual in the last, padded spectral rows between) against the oracle's
    FP64 iterates."""
    from janus_b200 import microstructures as micro
    from janus_b200 import operators as ops
    from janus_b200.solvers import BasicScheme
    phase = (micro.ellipses(max(shape), 4, seed=2)[:shape[0], :shape[1]] > 0).astype(np.uint8)
    pars = [O.delta_c(1.0, 0.3, 5.5, 0.3, 2), O.delta_c(10.0, 0.25, 5.5, 0.3, 2)]
    tens = [ops.isotropic_4(a, b, 2) for a, b in pars]
    loc = ops.BlockDiagonalOperator2D.from_phases(phase, tens, dtype=torch.float32)
    g = truncated(material.create(5.5, 0.3, 2).green_operator(), shape, 1.0,
                  dtype=torch.float32)
    E = np.array([0.0, 0.0, 1.0])
    r = BasicScheme(g, loc).run(E, 10)
    eps_o, res_o, _ = O.basic_scheme(phase, [p[0] for p in pars], [p[1] for p in pars], 5.5,
                                     0.3, E, 10)
    eps = r.eps[0].double().cpu().numpy()
    assert np.abs(eps - eps_o).max() <= 1e-5 * np.abs(eps_o).max()
    np.testing.assert_allclose(r.residuals[:, 0], res_o, rtol=1e-3)


@pytest.mark.gpu
def test_batched_apply_and_fp32():
    rng = np.random.default_rng(8)
    shape = (32, 24, 16)
    x = rng.normal(size=(3,) + shape + (6,))
    g64 = filtered(material.create(MU, NU, 3).green_operator(), shape, 1.0)
    y = g64.apply_batch(torch.from_numpy(x).cuda()).cpu().numpy()
    for b in range(3):
        ref = O.green_apply(x[b], MU, NU, 1.0, "filtered")
        np.testing.assert_allclose(y[b], ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
    g32 = filtered(material.create(MU, NU, 3).green_operator(), shape, 1.0, dtype="float32")
    y32 = g32.apply(torch.from_numpy(x[0]).float().cuda()).double().cpu().numpy()
    ref = O.green_apply(x[0], MU, NU, 1.0, "filtered")
    assert np.abs(y32 - ref).max() <= 2e-6 * np.abs(ref).max()


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(1024, 1024), (512, 384), (768, 256)])
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
def test_long_axis_2d_fp32_apply(shape, variant):
    """2D FP32 grids whose axis-0 tiles need an even column count for the
    TMA box (the tile-width search skips widths of 24 or 72 bytes)."""
    import janus_b200.material.elastic.linear.isotropic as _mat
    from janus_b200.green import filtered as _filtered, truncated as _truncated
    from oracle import janus_oracle as _O
    f = _truncated if variant == "truncated" else _filtered
    g = f(_mat.create(0.75, 0.3, 2).green_operator(), shape, 1.0, dtype=torch.float32)
    rng = np.random.default_rng(9)
    x = rng.standard_normal(shape + (3,)).astype(np.float32)
    y = g.apply(torch.from_numpy(x).cuda()).double().cpu().numpy()
    ref = _O.green_apply(x.astype(np.float64), 0.75, 0.3, 1.0, variant)
    assert np.abs(y - ref).max() <= 2e-5 * np.abs(ref).max()
