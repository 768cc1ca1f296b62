"""Serial real-to-complex FFT objects on the GPU.

Mirrors ``janus.fft.serial`` (janus/fft/serial/_serial_fft.pyx:20-325):
``create_real(shape, flags)`` returns an object with ``r2c``/``c2r`` and the
attributes ``ishape, oshape, global_ishape, global_oshape, isize, osize,
offset0, idispl, odispl``.  The complex layout is the reference's:
``oshape = (n0, [n1,] 2*(n_last//2 + 1))`` with real and imaginary parts
interleaved along the last axis.  ``r2c`` is unnormalised, ``c2r`` scales by
1/N (_serial_fft.pyx:74, 174-175).

Arrays may be numpy arrays (host, float64, any strides) or CUDA tensors.
"""
from __future__ import annotations

import ctypes

import numpy as np

from .. import _arrays as A
from .. import _lib

FFTW_MEASURE = 0
FFTW_DESTROY_INPUT = 1 << 0
FFTW_UNALIGNED = 1 << 1
FFTW_CONSERVE_MEMORY = 1 << 2
FFTW_EXHAUSTIVE = 1 << 3
FFTW_PRESERVE_INPUT = 1 << 4
FFTW_PATIENT = 1 << 5
FFTW_ESTIMATE = 1 << 6
FFTW_WISDOM_ONLY = 1 << 21

_INVALID_REAL = "shape of real array must be {0} [was {1}]"
_INVALID_COMPLEX = "shape of complex array must be {0} [was {1}]"


def create_real(shape, flags=FFTW_MEASURE, dtype=None):
    """Return a new FFT object for real-to-complex transforms of `shape`.

    Same contract as janus.fft.serial.create_real (_serial_fft.pyx:20-33):
    ValueError unless len(shape) is 2 or 3.
    """
    if len(shape) == 2:
        return RealFFT2D(shape[0], shape[1], flags, dtype)
    elif len(shape) == 3:
        return RealFFT3D(shape[0], shape[1], shape[2], flags, dtype)
    raise ValueError('length of shape can be 2 or 3 (was {0})'.format(len(shape)))


class _RealFFT:
    def __init__(self, shape, flags, dtype):
        self._dtype = A.torch_dtype(dtype)
        n = tuple(int(v) for v in shape)
        self._dim = len(n)
        m2 = 2 * (n[-1] // 2 + 1)
        self._ishape = n
        self._oshape = n[:-1] + (m2,)
        self._handle = ctypes.c_void_p()
        L = _lib.lib()
        _lib.check(L.jb_fft_create(self._dim, _lib.i64_array(n), A.jb_dtype(self._dtype),
                                   int(flags), ctypes.byref(self._handle)))
        # planning rigour, read by the Green operators built on this transform
        self._flags = int(flags)

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().jb_fft_destroy(h)
            except Exception:
                pass
            self._handle = None

    # attributes of _serial_fft.pxd:10-51 (serial: offset0 = 0, local = global)
    ishape = property(lambda self: self._ishape)
    oshape = property(lambda self: self._oshape)
    global_ishape = property(lambda self: self._ishape)
    global_oshape = property(lambda self: self._oshape)
    isize = property(lambda self: int(np.prod(self._ishape)))
    osize = property(lambda self: int(np.prod(self._oshape)))
    offset0 = property(lambda self: 0)
    idispl = property(lambda self: 0)
    odispl = property(lambda self: 0)
    dtype = property(lambda self: self._dtype)

    def _check(self, a, expected, template):
        s = A.shape_of(a)
        if s != expected:
            raise ValueError(template.format(expected, s))

    def r2c(self, r, c=None):
        """Forward transform of r (shape ishape) into c (shape oshape)."""
        self._check(r, self._ishape, _INVALID_REAL)
        if c is not None:
            self._check(c, self._oshape, _INVALID_COMPLEX)
        strides = None
        if A.is_tensor(r) and r.device.type == "cuda" and r.dtype == self._dtype:
            rd = r
            strides = _lib.i64_array(r.stride())
        else:
            rd = A.to_device(r, self._dtype)
        out = A.Output(c, self._oshape, self._dtype, r)
        _lib.check(_lib.lib().jb_fft_r2c(self._handle, ctypes.c_void_p(rd.data_ptr()), strides,
                                         ctypes.c_void_p(out.target.data_ptr()),
                                         ctypes.c_void_p(A.stream_handle())))
        return out.finish()

    def c2r(self, c, r=None):
        """Inverse transform (scaled by 1/N) of c (oshape) into r (ishape)."""
        self._check(c, self._oshape, _INVALID_COMPLEX)
        if r is not None:
            self._check(r, self._ishape, _INVALID_REAL)
        cd = A.to_device(c, self._dtype)
        out = A.Output(r, self._ishape, self._dtype, c)
        _lib.check(_lib.lib().jb_fft_c2r(self._handle, ctypes.c_void_p(cd.data_ptr()),
                                         ctypes.c_void_p(out.target.data_ptr()), None,
                                         ctypes.c_void_p(A.stream_handle())))
        return out.finish()


class RealFFT2D(_RealFFT):
    """2D real FFT (the reference's _RealFFT2D, _serial_fft.pyx:55-177)."""

    def __init__(self, n0, n1, flags=FFTW_MEASURE, dtype=None):
        super().__init__((n0, n1), flags, dtype)


class RealFFT3D(_RealFFT):
    """3D real FFT (the reference's _RealFFT3D, _serial_fft.pyx:179-325)."""

    def __init__(self, n0, n1, n2, flags=FFTW_MEASURE, dtype=None):
        super().__init__((n0, n1, n2), flags, dtype)


_RealFFT2D = RealFFT2D
_RealFFT3D = RealFFT3D
