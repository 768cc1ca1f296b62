"""The axis-0 Green pass whose transforms and contraction run in registers
(five-phase tiles for n0 = 32 ... 256, seven-phase tiles for 192, 384, 512,
768 and 1024, with 3-, 6-, 8-, 12- and 16-point first phases),
against the oracle and against the shared-memory column kernel, for the
three discretisations of janus/green.pyx (truncated 393-580, filtered
583-973 through the generic c_apply 185-216 / 356-390, finite differences
976-1036).

Shapes are chosen so that the last tile of the pass is ragged (coefficient
counts that do not fill the last tile, odd load-case counts), which the
kernel masks."""
import numpy as np
import pytest
import torch

import janus_b200.material.elastic.linear.isotropic as material
from janus_b200 import autotune
from janus_b200.green import filtered, truncated, willot2015
from oracle import janus_oracle as O

MU = 0.75
NU = 0.3
FACTORY = {"truncated": truncated, "filtered": filtered, "willot": willot2015}
# n0 from 32 to 1024 (five-phase tiles up to 256, seven-phase above); ragged
# coefficient counts in the last tile
SHAPES = [(128, 6, 10), (128, 5, 4), (64, 5, 8), (32, 9, 6), (192, 3, 6), (256, 3, 6),
          (384, 2, 6), (512, 2, 4), (768, 2, 4), (1024, 1, 6), (128, 18), (64, 7), (32, 33),
          (192, 12), (256, 10), (384, 9), (512, 6), (768, 10), (1024, 14)]
# register-tile Green pass (compile-time value 3), the contraction by the
# built-in rule
R4 = [0, 0, 1, 0, 0, 3, 0]


def _old_kernel(shape):
    """The shared-memory compile-time column kernel (12-column tiles)."""
    return [0, 0, 1, 12, 2, 1, 0]


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered", "willot"])
@pytest.mark.parametrize("shape", SHAPES)
@pytest.mark.parametrize("nload", [1, 3, 6])
def test_r4_green_pass_vs_oracle(variant, shape, nload):
    rng = np.random.default_rng(5 + nload)
    s = 3 if len(shape) == 2 else 6
    x = rng.normal(size=(nload,) + shape + (s,))
    g = FACTORY[variant](material.create(MU, NU, len(shape)).green_operator(), shape, 0.5)
    autotune.set_tuning(g, R4)
    xt = torch.from_numpy(x).cuda()
    y = g.apply_batch(xt).cpu().numpy()
    for l in range(nload):
        ref = O.green_apply(x[l], MU, NU, 0.5, variant)
        np.testing.assert_allclose(y[l], ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max(),
                                   err_msg=f"load case {l}")
    # the shared-memory kernel gives the same field to rounding
    autotune.set_tuning(g, _old_kernel(shape))
    y_old = g.apply_batch(xt).cpu().numpy()
    np.testing.assert_allclose(y, y_old, rtol=0, atol=1e-14 * np.abs(y_old).max())
    # in place
    autotune.set_tuning(g, R4)
    out = g.apply_batch(xt, xt)
    assert out is xt
    np.testing.assert_array_equal(xt.cpu().numpy(), y)


@pytest.mark.gpu
@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("shape", [(128, 6, 10), (128, 18)])
def test_r4_table_and_on_the_fly(mode, shape):
    """Truncated operator through the table (mode 1) and on the fly (mode 2)."""
    rng = np.random.default_rng(3)
    s = 3 if len(shape) == 2 else 6
    x = rng.normal(size=(2,) + shape + (s,))
    g = truncated(material.create(MU, NU, len(shape)).green_operator(), shape, 1.0)
    autotune.set_tuning(g, R4[:6] + [mode])
    y = g.apply_batch(torch.from_numpy(x).cuda()).cpu().numpy()
    for l in range(2):
        ref = O.green_apply(x[l], MU, NU, 1.0, "truncated")
        np.testing.assert_allclose(y[l], ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
@pytest.mark.parametrize("shape", [(128, 10, 12), (64, 33), (256, 4, 6), (1024, 10)])
def test_r4_fp32(variant, shape):
    """FP32 fields through the same pass: within FP32 rounding of the FP64 oracle."""
    rng = np.random.default_rng(9)
    s = 3 if len(shape) == 2 else 6
    x = rng.normal(size=(3,) + shape + (s,))
    g = FACTORY[variant](material.create(MU, NU, len(shape)).green_operator(), shape, 1.0,
                         dtype=torch.float32)
    autotune.set_tuning(g, R4)
    y = g.apply_batch(torch.from_numpy(x).float().cuda()).double().cpu().numpy()
    for l in range(3):
        ref = O.green_apply(x[l], MU, NU, 1.0, variant)
        assert np.abs(y[l] - ref).max() <= 2e-5 * np.abs(ref).max()
