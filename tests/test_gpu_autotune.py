"""Column-pass schedules: every candidate of the autotuner computes the same
Green operator, and the tuner picks, sets and caches one."""
import numpy as np
import pytest
import torch

import janus_b200.material.elastic.linear.isotropic as material
from janus_b200 import autotune
from janus_b200 import operators as ops
from janus_b200.green import filtered, truncated
from oracle import janus_oracle as O


def _green(dim, n, variant, dtype):
    mat = material.create(0.75, 0.3, dim)
    f = filtered if variant == "filtered" else truncated
    shape = (n,) * dim if np.isscalar(n) else tuple(n)
    return f(mat.green_operator(), shape, 1.0, dtype=dtype)


@pytest.mark.gpu
@pytest.mark.parametrize("dim,n,dtype", [(3, 32, torch.float64), (3, 64, torch.float32),
                                         (2, 64, torch.float64), (2, 96, torch.float32),
                                         (2, 256, torch.float64),
                                         (3, (256, 16, 16), torch.float64),
                                         (3, (256, 16, 16), torch.float32),
                                         (3, (128, 16, 16), torch.float64),
                                         (3, (128, 16, 16), torch.float32),
                                         (2, (128, 64), torch.float64),
                                         (2, (128, 62), torch.float32)])
def test_every_candidate_computes_the_same_operator(dim, n, dtype):
    g = _green(dim, n, "filtered", dtype)
    s = g.ishape[-1]
    rng = np.random.default_rng(0)
    x = torch.from_numpy(rng.standard_normal(tuple(g.ishape))).to("cuda", dtype)
    ref = g.apply(x).double().cpu().numpy()
    exact = O.green_apply(x.double().cpu().numpy(), 0.75, 0.3, 1.0, "filtered")
    tol = 1e-12 if dtype == torch.float64 else 2e-5
    plain, green = autotune.candidates(dim, dtype)
    base = autotune.get_tuning(g)
    for c in plain:
        autotune.set_tuning(g, list(c) + base[3:6])
        y = g.apply(x).double().cpu().numpy()
        assert np.abs(y - ref).max() <= tol * np.abs(ref).max(), c
    for mode in (1, 2):   # M/N table, on the fly
        for c in green:
            autotune.set_tuning(g, base[0:3] + list(c) + [mode])
            y = g.apply(x).double().cpu().numpy()
            assert np.abs(y - exact).max() <= tol * np.abs(exact).max(), (c, mode)


@pytest.mark.gpu
def test_tuning_validation():
    g = _green(3, 16, "truncated", torch.float64)
    with pytest.raises(ValueError):
        autotune.set_tuning(g, [8, 2, 1, 7, 2, 1])   # Green width not a multiple of 6
    with pytest.raises(ValueError):
        autotune.set_tuning(g, [8, 4, 1, 12, 2, 1])  # 4 input tiles
    autotune.set_tuning(g, [16, 3, 0, 18, 2, 1])
    assert autotune.get_tuning(g) == [16, 3, 0, 18, 2, 1, 0]
    autotune.set_tuning(g, [16, 3, 0, 18, 2, 1, 2])
    assert autotune.get_tuning(g) == [16, 3, 0, 18, 2, 1, 2]
    with pytest.raises(ValueError):
        autotune.set_tuning(g, [8, 2, 1, 12, 2, 1, 3])


@pytest.mark.gpu
@pytest.mark.parametrize("dim", [2, 3])
def test_tune_sets_and_caches(dim, tmp_path, monkeypatch):
    monkeypatch.setenv("JB_TUNE_CACHE", str(tmp_path / "tune.json"))
    n = 32 if dim == 3 else 128
    g = _green(dim, n, "filtered", torch.float64)
    phase = (np.indices((n,) * dim).sum(axis=0) % 3 == 0).astype(np.uint8)
    pars = [O.delta_c(1.0, 0.3, 5.5, 0.3, dim), O.delta_c(10.0, 0.3, 5.5, 0.3, dim)]
    tens = [ops.isotropic_4(a, b, dim) for a, b in pars]
    cls = ops.BlockDiagonalOperator3D if dim == 3 else ops.BlockDiagonalOperator2D
    loc = cls.from_phases(phase, tens)
    r1 = autotune.tune(g, loc, nload=2, steps=2, warmup=1)
    assert not r1["cached"]
    assert autotune.get_tuning(g) == r1["tuning"]
    plain, green = autotune.candidates(dim, torch.float64)
    assert tuple(r1["tuning"][3:6]) in green and r1["tuning"][6] in (1, 2)
    if dim == 3:
        assert tuple(r1["tuning"][0:3]) in plain
    g2 = _green(dim, n, "filtered", torch.float64)
    r2 = autotune.tune(g2, loc, nload=2)
    assert r2["cached"] and r2["tuning"] == r1["tuning"]
    assert autotune.get_tuning(g2) == r1["tuning"]
