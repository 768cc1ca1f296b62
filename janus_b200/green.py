"""Discrete Green operators for strains (the ``janus.green`` module).

Mirrors janus/green.pyx:22-1036 for the truncated, filtered and
finite-difference (Willot 2015) discretisations, 2D and 3D:

* ``truncated(green, n, h, transform=None)`` / ``filtered(...)`` (22-36),
  ``willot2015(...)`` (1030-1036);
* ``set_frequency(b)`` with the reference's range checks (146-163,
  312-334), ``to_memoryview(out)`` (165-171, 336-342), ``apply_by_freq(tau,
  eta)`` (173-180, 344-351): per-index host calls evaluated by the native
  library with the reference's formulas;
* ``apply(x, y=None)`` (the fused FFT -> Gamma-hat -> inverse FFT of
  185-216, 356-390, 456-495, 534-580): the sm_100a pass kernels, in place
  allowed, x and y numpy arrays or CUDA tensors.

``transform`` may be None: unlike the reference (whose apply needs an FFT
object), the GPU operator owns its transform plan, so apply works either
way; a given transform must have ``global_ishape == n`` (green.pyx:115-118),
and its planner flags choose how the column passes are scheduled on first
use (see ``janus_b200.fft``).
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _arrays as A
from . import _lib
from .material.elastic.linear.isotropic import _GreenOperatorForStrains
from .operators import (AbstractStructuredOperator2D, AbstractStructuredOperator3D,
                        _check_1d, _out_1d, _out_2d)

_P = ctypes.POINTER(ctypes.c_double)
_PI = ctypes.POINTER(ctypes.c_int32)


def truncated(green, n, h, transform=None, dtype=None):
    """Truncated discrete Green operator (green.pyx:22-28)."""
    if green.dim == 2:
        return TruncatedGreenOperator2D(green, n, h, transform, dtype)
    elif green.dim == 3:
        return TruncatedGreenOperator3D(green, n, h, transform, dtype)
    raise ValueError('dim must be 2 or 3 (was {0})'.format(green.dim))


def filtered(green, n, h, transform=None, dtype=None):
    """Filtered discrete Green operator (green.pyx:30-36)."""
    if green.dim == 2:
        return FilteredGreenOperator2D(green, n, h, transform, dtype)
    elif green.dim == 3:
        return FilteredGreenOperator3D(green, n, h, transform, dtype)
    raise ValueError('dim must be 2 or 3 (was {0})'.format(green.dim))


def willot2015(green, n, h, transform=None, dtype=None):
    """Finite-difference ("rotated scheme", Willot 2015) discrete Green
    operator (green.pyx:1030-1036): Gamma0 at the modified wave-vector
    k_i = sin(phi_i) prod_{j != i} cos(phi_j), phi_i = pi b_i / n_i."""
    if green.dim == 2:
        return FiniteDifferences2D(green, n, h, transform, dtype)
    elif green.dim == 3:
        return FiniteDifferences3D(green, n, h, transform, dtype)
    raise ValueError('dim must be 2 or 3 (was {0})'.format(green.dim))


class _DiscreteGreenOperator:
    _variant = None

    def _setup(self, green, shape, h, transform, dtype):
        dim = self._ndim
        if len(shape) != dim:
            raise ValueError('length of shape must be {0} (was {1})'.format(dim, len(shape)))
        if not isinstance(green, _GreenOperatorForStrains) or green.dim != dim:
            raise ValueError('continuous green operator must operate in '
                             'a {0}D space'.format(dim))
        h = float(h)
        if h <= 0.:
            raise ValueError('h must be > 0 (was {0})'.format(h))
        shape = tuple(int(v) for v in shape)
        if transform is not None:
            if tuple(transform.global_ishape) != shape:
                raise ValueError('shape of transform must be {0} [was {1}]'.format(
                    shape, transform.global_ishape))
        if dtype is None and transform is not None:
            dtype = transform.dtype
        self._dtype = A.torch_dtype(dtype)
        self._green = green
        self._h = h
        self._transform = transform
        self.init_shapes(*shape, green.isize, green.osize)
        # schedule of the column passes, chosen on first use per batch size
        # by the transform's planning rigour (janus_b200.fft); FFTW_MEASURE
        # when no transform is given, as the reference's create_real default
        self._planning = int(getattr(transform, "_flags", 0)) if transform is not None else 0
        self._planned = set()
        self._handle = ctypes.c_void_p()
        mat = green.mat
        _lib.check(_lib.lib().jb_green_create(
            dim, _lib.i64_array(shape), h, mat.g, mat.nu, self._variant,
            A.jb_dtype(self._dtype), ctypes.byref(self._handle)))
        self._b = None
        self._matrix = None

    def __del__(self):
        hd = getattr(self, "_handle", None)
        if hd is not None and hd.value:
            try:
                _lib.lib().jb_green_destroy(hd)
            except Exception:
                pass
            self._handle = None

    green = property(lambda self: self._green)
    h = property(lambda self: self._h)
    transform = property(lambda self: self._transform)
    dtype = property(lambda self: self._dtype)

    @property
    def handle(self):
        return self._handle

    def set_frequency(self, b):
        """Select the discrete frequency b (ints, 0 <= b_i < n_i)."""
        b = np.asarray(b)
        if b.ndim != 1 or b.shape[0] != self._ndim:
            raise ValueError('invalid shape: expected ({0},), actual ({1},)'.format(
                self._ndim, b.shape[0] if b.ndim == 1 else b.shape))
        bb = np.ascontiguousarray(b, dtype=np.int32)
        m = np.empty((self.oshape[-1], self.ishape[-1]))
        _lib.check(_lib.lib().jb_green_matrix(self._handle, bb.ctypes.data_as(_PI),
                                              m.ctypes.data_as(_P)))
        self._b = bb
        self._matrix = m

    def to_memoryview(self, out=None):
        out = _out_2d(out, self.oshape[-1], self.ishape[-1])
        if self._matrix is None:
            raise ValueError('set_frequency() must be called first')
        out[...] = self._matrix
        return out[...]

    def apply_by_freq(self, tau, eta=None):
        tau = np.ascontiguousarray(np.asarray(tau, dtype=np.float64))
        _check_1d(tau, self.ishape[-1])
        eta = _out_1d(eta, self.oshape[-1])
        if self._b is None:
            raise ValueError('set_frequency() must be called first')
        res = np.empty(self.oshape[-1])
        _lib.check(_lib.lib().jb_green_apply_by_freq(self._handle, self._b.ctypes.data_as(_PI),
                                                     tau.ctypes.data_as(_P),
                                                     res.ctypes.data_as(_P)))
        eta[...] = res
        return eta[...]

    def apply_by_freq_device(self, b, tau, eta=None):
        """Green contraction on the GPU at many indices at once.

        b: int32 (count, dim); tau: complex (count, s) as a (count, s, 2) real
        CUDA tensor.  Runs the same device code as apply()."""
        if A.is_tensor(b):
            bd = b.to(A.device()).to(torch.int32).contiguous()
        else:
            bd = torch.from_numpy(np.ascontiguousarray(np.asarray(b, dtype=np.int32))).to(
                A.device())
        if bd.ndim != 2 or bd.shape[1] != self._ndim:
            raise ValueError('b must have shape (count, {0})'.format(self._ndim))
        if bd.shape[0]:
            lo = bd.min(dim=0).values.cpu().numpy()
            hi = bd.max(dim=0).values.cpu().numpy()
            for d in range(self._ndim):
                if lo[d] < 0 or hi[d] >= self.ishape[d]:
                    raise ValueError('index must be >= 0 and < {0}'.format(self.ishape[d]))
        td = A.to_device(tau, self._dtype)
        if tuple(td.shape) != (bd.shape[0], self.ishape[-1], 2):
            raise ValueError('tau must have shape (count, {0}, 2)'.format(self.ishape[-1]))
        if eta is None:
            eta = td.clone()
        _lib.check(_lib.lib().jb_green_apply_by_freq_device(
            self._handle, int(bd.shape[0]), ctypes.c_void_p(bd.data_ptr()),
            ctypes.c_void_p(td.data_ptr()), ctypes.c_void_p(eta.data_ptr()),
            ctypes.c_void_p(A.stream_handle())))
        return eta

    def _plan(self, nload):
        """FFTW_ESTIMATE: the built-in schedule rule; FFTW_MEASURE and
        FFTW_WISDOM_ONLY: the autotuner's cached schedule if any;
        FFTW_PATIENT / FFTW_EXHAUSTIVE: run the autotuner once (cached)."""
        if nload in self._planned:
            return
        self._planned.add(nload)
        from .fft.serial import FFTW_ESTIMATE, FFTW_EXHAUSTIVE, FFTW_PATIENT
        if self._planning & FFTW_ESTIMATE:
            return
        from . import autotune
        if self._planning & (FFTW_PATIENT | FFTW_EXHAUSTIVE):
            autotune.tune(self, None, nload=nload)
        else:
            autotune.apply_cached(self, nload)

    def _apply_device(self, x, y):
        self._plan(1)
        _lib.check(_lib.lib().jb_green_apply(self._handle, ctypes.c_void_p(x.data_ptr()),
                                             ctypes.c_void_p(y.data_ptr()), 1,
                                             ctypes.c_void_p(A.stream_handle())))

    def apply_batch(self, x, y=None):
        """Apply to a batch of fields (CUDA tensor of shape (B,) + ishape)."""
        if not A.is_tensor(x) or tuple(x.shape[1:]) != self.ishape:
            raise ValueError('expected a CUDA tensor of shape (B,) + {0}'.format(self.ishape))
        xd = A.to_device(x, self._dtype)
        if y is None:
            y = xd.new_empty(xd.shape)
        self._plan(int(xd.shape[0]))
        _lib.check(_lib.lib().jb_green_apply(self._handle, ctypes.c_void_p(xd.data_ptr()),
                                             ctypes.c_void_p(y.data_ptr()), int(xd.shape[0]),
                                             ctypes.c_void_p(A.stream_handle())))
        return y


class DiscreteGreenOperator2D(_DiscreteGreenOperator, AbstractStructuredOperator2D):
    def __init__(self, green, shape, h, transform=None, dtype=None):
        AbstractStructuredOperator2D.__init__(self)
        self._setup(green, shape, h, transform, dtype)


class DiscreteGreenOperator3D(_DiscreteGreenOperator, AbstractStructuredOperator3D):
    def __init__(self, green, shape, h, transform=None, dtype=None):
        AbstractStructuredOperator3D.__init__(self)
        self._setup(green, shape, h, transform, dtype)


class TruncatedGreenOperator2D(DiscreteGreenOperator2D):
    """green.pyx:393-495"""
    _variant = _lib.JB_TRUNCATED


class TruncatedGreenOperator3D(DiscreteGreenOperator3D):
    """green.pyx:498-580"""
    _variant = _lib.JB_TRUNCATED


class FilteredGreenOperator2D(DiscreteGreenOperator2D):
    """green.pyx:583-694"""
    _variant = _lib.JB_FILTERED


class FilteredGreenOperator3D(DiscreteGreenOperator3D):
    """green.pyx:697-973"""
    _variant = _lib.JB_FILTERED


class FiniteDifferences2D(DiscreteGreenOperator2D):
    """green.pyx:976-992"""
    _variant = _lib.JB_WILLOT


class FiniteDifferences3D(DiscreteGreenOperator3D):
    """green.pyx:995-1027"""
    _variant = _lib.JB_WILLOT
