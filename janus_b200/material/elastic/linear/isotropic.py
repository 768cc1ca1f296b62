"""Isotropic, linear elastic materials and their Green operator for strains.

Mirrors ``janus.material.elastic.linear.isotropic``
(janus/material/elastic/linear/isotropic.pyx:23-353): ``create(g, nu, dim)``,
``poisson_from_bulk_and_shear_moduli``, the material's read-only ``g, nu, k,
dim`` and ``green_operator()``, whose ``set_frequency(k)``, ``apply(x, y)``
and ``to_memoryview(out)`` act on one wave-vector.  Those per-wave-vector
calls evaluate the reference's formulas in the native library (host code,
same operations); the field-wide application of the operator is
``janus_b200.green``.

dim == 2 is plane strain; a plane-stress material with (g, nu) is the
plane-strain one with (g, nu / (1 + nu)) (isotropic.pyx:10-12).
"""
from __future__ import annotations

import ctypes

import numpy as np

from ...._lib import check, lib
from ....operators import AbstractLinearOperator, _check_1d, _out_1d, _out_2d


def create(g, nu, dim=3):
    """Return a new IsotropicLinearElasticMaterial (isotropic.pyx:23-29)."""
    return IsotropicLinearElasticMaterial(g, nu, dim)


def poisson_from_bulk_and_shear_moduli(k, g, dim=3):
    """Poisson ratio from bulk and shear moduli (isotropic.pyx:32-46)."""
    k = float(k)
    g = float(g)
    if dim == 2:
        return (k - g) / (2. * k)
    elif dim == 3:
        return (3 * k - 2 * g) / (2 * (3 * k + g))
    raise ValueError('dim must be 2 or 3 (was {0})'.format(dim))


class IsotropicLinearElasticMaterial:
    """Isotropic linear elastic material (isotropic.pyx:49-96).

    Attributes ``g`` (shear modulus), ``nu`` (Poisson ratio), ``k`` (bulk
    modulus; plane strain in 2D) and ``dim`` are read-only.
    """

    __slots__ = ("_g", "_nu", "_k", "_dim")

    def __init__(self, g, nu, dim=3):
        g = float(g)
        nu = float(nu)
        dim = int(dim)
        # validation of isotropic.pyx:63-70
        if g < 0.0:
            raise ValueError('g must be >= 0 (was {0})'.format(g))
        if dim == 2 and nu > 0.5:
            raise ValueError('nu must be <= 1/2 (was {0})'.format(nu))
        if dim == 3 and (nu < -1.0 or nu > 0.5):
            raise ValueError('nu must be >= -1 and <= 1/2 (was {0})'.format(nu))
        if dim != 2 and dim != 3:
            raise ValueError('dim must be 2 or 3 (was {0})'.format(dim))
        object.__setattr__(self, "_g", g)
        object.__setattr__(self, "_nu", nu)
        object.__setattr__(self, "_dim", dim)
        if dim == 2:
            k = g / (1. - 2. * nu)
        else:
            k = 2. / 3. * (1. + nu) / (1. - 2. * nu) * g
        object.__setattr__(self, "_k", k)

    g = property(lambda self: self._g)
    nu = property(lambda self: self._nu)
    k = property(lambda self: self._k)
    dim = property(lambda self: self._dim)

    def __setattr__(self, name, value):
        raise AttributeError("attribute '{0}' of IsotropicLinearElasticMaterial "
                             "objects is not writable".format(name))

    def __repr__(self):
        return ('IsotropicLinearElasticMaterial'
                '(g={0}, nu={1}, dim={2})').format(self.g, self.nu, self.dim)

    def green_operator(self):
        """Periodic Green operator for strains of this material."""
        if self.dim == 2:
            return GreenOperatorForStrains2D(self)
        return GreenOperatorForStrains3D(self)


class _GreenOperatorForStrains(AbstractLinearOperator):
    """Continuous Green operator for strains (isotropic.pyx:99-138)."""

    _expected_dim = None

    def __init__(self, mat):
        if not isinstance(mat, IsotropicLinearElasticMaterial):
            raise TypeError("mat must be an IsotropicLinearElasticMaterial")
        if mat.dim != self._expected_dim:
            raise ValueError('plane strain material expected' if self._expected_dim == 2
                             else '3D material expected')
        sym = (mat.dim * (mat.dim + 1)) // 2
        super().__init__()
        self.init_sizes(sym, sym)
        self._mat = mat
        self._dim = mat.dim
        self._matrix = np.zeros((sym, sym))
        self._k = np.zeros(mat.dim)

    mat = property(lambda self: self._mat)
    dim = property(lambda self: self._dim)

    def __repr__(self):
        return 'Green Operator({0})'.format(self.mat)

    def set_frequency(self, k):
        """Set the wave-vector of subsequent apply/to_memoryview calls
        (green.pyx:69-83 with isotropic.pyx:158-182, 227-290)."""
        k = np.ascontiguousarray(np.asarray(k, dtype=np.float64))
        _check_1d(k, self.dim)
        out = np.zeros((self.osize, self.isize))
        check(lib().jb_green_continuous_matrix(
            self.dim, self._mat.g, self._mat.nu,
            k.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))
        self._k = k.copy()
        self._matrix = out

    def apply(self, x, y=None):
        """y = Gamma(k) x (isotropic.pyx:186-193, 294-313)."""
        x = np.ascontiguousarray(np.asarray(x, dtype=np.float64))
        _check_1d(x, self.isize)
        y = _out_1d(y, self.osize)
        res = np.empty(self.osize)
        P = ctypes.POINTER(ctypes.c_double)
        check(lib().jb_green_continuous_apply(
            self.dim, self._mat.g, self._mat.nu, self._k.ctypes.data_as(P),
            x.ctypes.data_as(P), res.ctypes.data_as(P)))
        y[...] = res
        return y[...]

    def to_memoryview(self, out=None):
        out = _out_2d(out, self.osize, self.isize)
        out[...] = self._matrix
        return out[...]


class GreenOperatorForStrains2D(_GreenOperatorForStrains):
    _expected_dim = 2


class GreenOperatorForStrains3D(_GreenOperatorForStrains):
    _expected_dim = 3


_GreenOperatorForStrains2D = GreenOperatorForStrains2D
_GreenOperatorForStrains3D = GreenOperatorForStrains3D
