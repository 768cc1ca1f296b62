"""CPU tests of the native library: it loads, exports every entry point the
public header declares, and its host-side per-vector functions follow the
reference exactly.  No GPU compute is called here."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import janus_oracle as O
from tests.conftest import ROOT, ULP


def _declared_functions():
    text = open(os.path.join(ROOT, "include", "janus_b200.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(jb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from janus_b200 import _lib
    L = _lib.lib()
    names = _declared_functions()
    assert len(names) >= 20
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    assert L.jb_version() >= 100
    assert L.jb_max_axis_length(0) >= 1024


@pytest.mark.parametrize("dim", [2, 3])
def test_continuous_matrix_is_the_reference_formula(dim):
    from janus_b200.material.elastic.linear import isotropic as mat
    rng = np.random.default_rng(3)
    g = mat.create(0.7, 0.3, dim).green_operator()
    for _ in range(40):
        k = rng.normal(size=dim) * 2.5
        g.set_frequency(k)
        np.testing.assert_array_equal(g.to_memoryview(), O.green_matrix(k, 0.7, 0.3))
        x = rng.normal(size=g.isize)
        np.testing.assert_allclose(g.apply(x), O.green_matrix(k, 0.7, 0.3) @ x, rtol=4 * ULP,
                                   atol=4 * ULP)
    g.set_frequency(np.zeros(dim))
    assert not np.asarray(g.to_memoryview()).any()


def test_green_operator_call_forms():
    from janus_b200.material.elastic.linear import isotropic as mat
    g = mat.create(0.7, 0.3, 3).green_operator()
    g.set_frequency(np.array([1., 2., 3.]))
    tau = np.zeros(6)
    tau[2] = 1.0
    expected = np.asarray(g.apply(tau)).copy()
    base = np.empty(6)
    out = g.apply(tau, base)
    assert out.base is base
    out = g.apply(tau, tau)
    assert out.base is tau
    np.testing.assert_array_equal(tau, expected)
    with pytest.raises(ValueError):
        g.set_frequency(np.zeros(4))


def test_materials_known_answer():
    # sphinx/materials.rst:54-68: Gamma at k=(1,2,3), mu=1, nu=0.3, Mandel
    from janus_b200.material.elastic.linear import isotropic as mat
    g = mat.create(1.0, 0.3, 3).green_operator()
    k = np.array([1., 2., 3.])
    g.set_frequency(k)
    np.testing.assert_array_equal(g.to_memoryview(), O.green_matrix(k, 1.0, 0.3))


@pytest.mark.parametrize("g, nu, dim", [(2.0, 0.3, 2), (2.0, 0.3, 3)])
def test_poisson_from_bulk_and_shear(g, nu, dim):
    from janus_b200.material.elastic.linear import isotropic as mat
    m = mat.create(g, nu, dim)
    assert mat.poisson_from_bulk_and_shear_moduli(m.k, g, dim) == nu


@pytest.mark.parametrize("g, k, nu, dim", [(1.5, 3.75, 0.3, 2), (1.5, 3.25, 0.3, 3)])
def test_material_init(g, k, nu, dim):
    from janus_b200.material.elastic.linear import isotropic as mat
    m = mat.create(g, nu, dim)
    assert (m.g, m.k, m.nu) == (g, k, nu)


@pytest.mark.parametrize("g, nu, dim", [(-1.0, 0.3, 2), (-1.0, 0.3, 3), (1.0, 0.5 + 1e-14, 2),
                                        (1.0, 1.0, 2), (1.0, -1.0 - 1e-14, 3), (1.0, -1.5, 3),
                                        (1.0, 0.5 + 1e-14, 3), (1.0, 1.0, 3), (1.0, 0.3, 0),
                                        (1.0, 0.3, 4)])
def test_material_invalid(g, nu, dim):
    from janus_b200.material.elastic.linear import isotropic as mat
    with pytest.raises(ValueError):
        mat.create(g, nu, dim)


@pytest.mark.parametrize("name, value", [("g", 2.0), ("k", 10.0), ("nu", 0.5), ("dim", 2)])
def test_material_read_only(name, value):
    from janus_b200.material.elastic.linear import isotropic as mat
    m = mat.create(1.0, 0.3, 3)
    with pytest.raises(AttributeError):
        setattr(m, name, value)


@pytest.mark.parametrize("dim", [2, 3])
def test_isotropic_tensor_exact(dim):
    from janus_b200.operators import isotropic_4
    rng = np.random.default_rng(7)
    for _ in range(20):
        sph, dev = rng.uniform(-3, 3, size=2)
        t = isotropic_4(sph, dev, dim)
        x = rng.normal(size=t.isize)
        np.testing.assert_array_equal(t.apply(x), O.isotropic_apply(x, sph, dev, dim))
        m = np.asarray(t.to_memoryview())
        np.testing.assert_allclose(m @ x, t.apply(x), rtol=1e-14, atol=1e-14)
        xx = x.copy()
        out = t.apply(xx, xx)
        assert out.base is xx


def test_isotropic_4_invalid_dim():
    from janus_b200.operators import isotropic_4
    with pytest.raises(ValueError):
        isotropic_4(1.0, 1.0, 4)


def test_abstract_operator_sizes():
    from janus_b200.operators import AbstractOperator
    op = AbstractOperator()
    op.init_sizes(4, 5)
    assert (op.isize, op.osize) == (4, 5)
    for a, b in [(0, 1), (-1, 1), (1, 0), (1, -1)]:
        with pytest.raises(ValueError):
            op.init_sizes(a, b)
    with pytest.raises(ValueError):
        op.apply(np.zeros(5))
    base = np.zeros(5)
    assert op.apply(np.zeros(4), base).base is base


def test_fft_create_real_invalid_rank():
    from janus_b200.fft import serial
    with pytest.raises(ValueError):
        serial.create_real((4,))
    with pytest.raises(ValueError):
        serial.create_real((4, 4, 4, 4))
