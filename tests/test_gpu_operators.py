"""Block-diagonal operators on the GPU against the oracle (bitwise for the
isotropic phase-map form, as the reference's per-voxel comparison in
tests/test_operators.py:447-450) and the reference's argument checks."""
import numpy as np
import pytest
import torch

from janus_b200 import operators as ops
from oracle import janus_oracle as O
from tests.conftest import ULP


def _phase_ops(shape, nphase, dim, seed=0):
    rng = np.random.default_rng(seed)
    phase = rng.integers(0, nphase, size=shape)
    sph = rng.uniform(-5, 5, size=nphase)
    dev = rng.uniform(-5, 5, size=nphase)
    tens = [ops.isotropic_4(a, b, dim) for a, b in zip(sph, dev)]
    loc = np.empty(shape, dtype=object)
    for idx in np.ndindex(*shape):
        loc[idx] = tens[phase[idx]]
    return phase, sph, dev, loc


@pytest.mark.gpu
@pytest.mark.parametrize("shape", [(7, 9), (16, 16), (5, 6, 7), (8, 8, 8)])
@pytest.mark.parametrize("nphase", [1, 3, 300])
def test_block_diagonal_isotropic_bitwise(shape, nphase):
    dim = len(shape)
    phase, sph, dev, loc = _phase_ops(shape, nphase, dim)
    op = ops.block_diagonal_operator(loc)
    assert op.local is not None
    s = 3 if dim == 2 else 6
    x = np.random.default_rng(1).normal(size=shape + (s,))
    y = np.asarray(op.apply(x))
    np.testing.assert_array_equal(y, O.phase_apply(x, phase, sph, dev, dim))
    # each voxel equals the single-vector local operator
    for idx in list(np.ndindex(*shape))[:20]:
        np.testing.assert_array_equal(y[idx], loc[idx].apply(x[idx]))
    base = np.zeros_like(x)
    assert op.apply(x, base).base is base
    xt = torch.from_numpy(x).cuda()
    assert op.apply(xt, xt) is xt
    np.testing.assert_array_equal(xt.cpu().numpy(), y)


@pytest.mark.gpu
def test_block_diagonal_from_phases():
    shape = (12, 10, 8)
    phase, sph, dev, _ = _phase_ops(shape, 2, 3, seed=3)
    tens = [ops.isotropic_4(a, b, 3) for a, b in zip(sph, dev)]
    op = ops.BlockDiagonalOperator3D.from_phases(phase, tens)
    x = np.random.default_rng(2).normal(size=shape + (6,))
    np.testing.assert_array_equal(np.asarray(op.apply(x)), O.phase_apply(x, phase, sph, dev, 3))


@pytest.mark.gpu
def test_block_diagonal_general_linear_local_ops():
    shape = (6, 5)
    rng = np.random.default_rng(4)
    mats = [rng.normal(size=(3, 3)) for _ in range(2)]

    class Mat(ops.AbstractLinearOperator):
        def __init__(self, m):
            super().__init__()
            self.init_sizes(3, 3)
            self.m = m

        def _to_matrix(self):
            return self.m
    tens = [Mat(m) for m in mats]
    phase = rng.integers(0, 2, size=shape)
    loc = np.empty(shape, dtype=object)
    for idx in np.ndindex(*shape):
        loc[idx] = tens[phase[idx]]
    op = ops.block_diagonal_operator(loc)
    x = rng.normal(size=shape + (3,))
    y = np.asarray(op.apply(x))
    for idx in np.ndindex(*shape):
        np.testing.assert_allclose(y[idx], mats[phase[idx]] @ x[idx], rtol=4 * ULP, atol=4 * ULP)


@pytest.mark.gpu
def test_block_diagonal_invalid():
    with pytest.raises(ValueError):
        ops.BlockDiagonalOperator2D(None)
    loc = np.empty((2, 2), dtype=object)
    loc[...] = ops.isotropic_4(1., 1., 2)
    loc[1, 1] = ops.isotropic_4(1., 1., 3)
    with pytest.raises(ValueError):
        ops.block_diagonal_operator(loc)
    loc[1, 1] = ops.isotropic_4(1., 1., 2)
    op = ops.block_diagonal_operator(loc)
    with pytest.raises(ValueError):
        op.apply(np.zeros((2, 2, 4)))
    with pytest.raises(ValueError):
        op.apply(np.zeros((2, 2, 3)), np.zeros((2, 3, 3)))


@pytest.mark.gpu
@pytest.mark.parametrize("shape, o, i", [((6, 7), 3, 3), ((4, 5), 2, 5), ((3, 4, 5), 6, 6),
                                         ((3, 2, 4), 4, 1)])
def test_block_diagonal_linear(shape, o, i):
    rng = np.random.default_rng(9)
    a = rng.normal(size=shape + (o, i))
    op = ops.block_diagonal_linear_operator(a)
    assert op.ishape == shape + (i,) and op.oshape == shape + (o,)
    x = rng.normal(size=shape + (i,))
    y = np.asarray(op.apply(x))
    np.testing.assert_array_equal(y, O.block_linear_apply(a, x))
    xt = rng.normal(size=shape + (o,))
    yt = np.asarray(op.apply_transpose(xt))
    np.testing.assert_array_equal(yt, O.block_linear_apply(a, xt, transpose=True))
    # adjoint identity <y, A x> = <A^T y, x> (tests/test_operators.py:506-509)
    assert abs(np.sum(xt * y) - np.sum(yt * x)) <= 1e-12 * np.abs(xt * y).sum()


@pytest.mark.gpu
def test_block_diagonal_linear_invalid():
    with pytest.raises(ValueError):
        ops.block_diagonal_linear_operator(np.zeros((2, 3, 4)))
    op = ops.block_diagonal_linear_operator(np.zeros((2, 3, 4, 5)))
    with pytest.raises(ValueError):
        op.apply(np.zeros((2, 3, 4)))
    with pytest.raises(ValueError):
        op.apply_transpose(np.zeros((2, 3, 5)))
