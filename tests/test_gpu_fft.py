"""GPU FFT objects against numpy's FFT, with the reference's own cases and
tolerances (tests/test_fft.py:9-80 of the reference)."""
import numpy as np
import pytest
import torch

from janus_b200.fft import serial

SHAPE_DELTA = [((256, 128), 2E-15), ((256, 129), 2E-14), ((257, 128), 2E-15),
               ((257, 129), 2E-14), ((128, 32, 64), 3E-15), ((127, 32, 64), 3E-15),
               ((128, 31, 64), 3.5E-15), ((128, 32, 63), 3.5E-15)]


def _rel_l1(actual, expected):
    return np.sum(np.abs(actual - expected)) / np.sum(np.abs(expected))


@pytest.mark.gpu
@pytest.mark.parametrize("shape, delta", SHAPE_DELTA)
@pytest.mark.parametrize("inplace", [True, False])
def test_r2c(shape, delta, inplace):
    transform = serial.create_real(shape)
    np.random.seed(20150312)
    a = 2. * np.random.rand(*transform.ishape) - 1.
    output = np.empty(transform.oshape, dtype=np.float64) if inplace else None
    output = np.asarray(transform.r2c(a, output))
    actual = output[..., 0::2] + 1j * output[..., 1::2]
    assert _rel_l1(actual, np.fft.rfftn(a)) <= delta


@pytest.mark.gpu
@pytest.mark.parametrize("shape, delta", SHAPE_DELTA)
@pytest.mark.parametrize("inplace", [True, False])
def test_c2r(shape, delta, inplace):
    transform = serial.create_real(shape)
    np.random.seed(20150312)
    expected = 2. * np.random.rand(*transform.ishape) - 1.
    a = np.asarray(transform.r2c(expected))
    if inplace:
        actual = transform.c2r(a, np.empty(transform.ishape, dtype=np.float64))
    else:
        actual = transform.c2r(a)
    assert _rel_l1(np.asarray(actual), expected) <= delta


INVALID = [((128, 256), (127, 256), (128, 258)), ((128, 256), (128, 255), (128, 258)),
           ((128, 256), (128, 256), (129, 258)), ((128, 256), (128, 256), (128, 259)),
           ((128, 64, 32), (127, 64, 32), (128, 64, 34)),
           ((128, 64, 32), (128, 63, 32), (128, 64, 34)),
           ((128, 64, 32), (128, 64, 31), (128, 64, 34)),
           ((128, 64, 32), (128, 64, 32), (127, 64, 34)),
           ((128, 64, 32), (128, 64, 32), (128, 63, 34)),
           ((128, 64, 32), (128, 64, 32), (128, 64, 33))]


@pytest.mark.gpu
@pytest.mark.parametrize("shape, ishape, oshape", INVALID)
@pytest.mark.parametrize("direct", [True, False])
def test_invalid_params(shape, ishape, oshape, direct):
    r = np.empty(ishape, dtype=np.float64)
    c = np.empty(oshape, dtype=np.float64)
    with pytest.raises(ValueError):
        if direct:
            serial.create_real(shape).r2c(r, c)
        else:
            serial.create_real(shape).c2r(c, r)


@pytest.mark.gpu
def test_attributes():
    t = serial.create_real((8, 9, 10))
    assert t.ishape == (8, 9, 10)
    assert t.oshape == (8, 9, 12)
    assert t.global_ishape == (8, 9, 10) and t.global_oshape == (8, 9, 12)
    assert (t.isize, t.osize, t.offset0, t.idispl, t.odispl) == (720, 864, 0, 0, 0)
    t = serial.create_real((7, 5))
    assert t.oshape == (7, 6)


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(64, 96), (1, 1), (2, 3), (3, 1, 5), (40, 50, 60),
                                   (200, 300), (11, 13, 17), (1024, 12), (5, 4096)])
def test_r2c_c2r_torch_sizes(shape):
    rng = np.random.default_rng(0)
    a = rng.uniform(-1, 1, size=shape)
    t = serial.create_real(shape)
    x = torch.from_numpy(a).cuda()
    c = t.r2c(x)
    assert isinstance(c, torch.Tensor) and c.is_cuda
    cn = c.cpu().numpy()
    exp = np.fft.rfftn(a)
    err = _rel_l1(cn[..., 0::2] + 1j * cn[..., 1::2], exp)
    assert err <= 5e-15
    back = t.c2r(c).cpu().numpy()
    assert _rel_l1(back, a) <= 5e-15
    # c2r leaves its input untouched
    np.testing.assert_array_equal(c.cpu().numpy(), cn)


@pytest.mark.gpu
def test_r2c_strided_tensor():
    rng = np.random.default_rng(1)
    big = torch.from_numpy(rng.uniform(-1, 1, size=(32, 24, 3))).cuda()
    t = serial.create_real((32, 24))
    c = t.r2c(big[:, :, 1]).cpu().numpy()
    exp = np.fft.rfftn(big[:, :, 1].cpu().numpy())
    assert _rel_l1(c[..., 0::2] + 1j * c[..., 1::2], exp) <= 5e-15


@pytest.mark.gpu
# (375, 40), (700, 24): column passes whose row count has no divisor up to
# 256 with 128-byte-aligned tensor-copy boxes (375) or only a smaller one
# (700: 140-row boxes rather than 175)
@pytest.mark.parametrize("shape", [(128, 128), (64, 32, 48), (96, 100), (375, 40), (700, 24)])
def test_fp32_transform(shape):
    rng = np.random.default_rng(2)
    a = rng.uniform(-1, 1, size=shape)
    t = serial.create_real(shape, dtype="float32")
    c = t.r2c(torch.from_numpy(a).float().cuda()).double().cpu().numpy()
    err = _rel_l1(c[..., 0::2] + 1j * c[..., 1::2], np.fft.rfftn(a))
    assert err <= 2e-6
