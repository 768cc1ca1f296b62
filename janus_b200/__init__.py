"""janus_b200: a B200-native implementation of Janus's FFT-based
Lippmann-Schwinger hot path.

The modules mirror the reference's (sbrisard/janus) API:

* ``janus_b200.fft.serial``       - ``create_real`` FFT objects (r2c / c2r)
* ``janus_b200.material.elastic.linear.isotropic`` - materials and the
  continuous Green operator for strains
* ``janus_b200.green``            - ``truncated`` / ``filtered`` discrete Green
  operators (2D/3D) with ``apply``, ``apply_by_freq``, ``set_frequency``
* ``janus_b200.operators``        - ``isotropic_4``, block-diagonal operators
* ``janus_b200.solvers``          - the basic fixed-point scheme

All field-wide work runs in hand-written sm_100a kernels behind the C ABI of
``include/janus_b200.h``; ``janus_b200.compat.install_as_janus()`` makes
existing ``import janus...`` scripts use this package.
"""
from . import _lib

__version__ = "0.1.0"


def native_library_path() -> str:
    """Path of the loaded native library (building it first if needed)."""
    _lib.lib()
    return _lib.library_path()
