"""Loader of the reference checker (test infrastructure only).

``load()`` imports the reference's own Cython modules compiled by
``oracle/build_ref.py`` into ``oracle/_ref`` (package name ``janus``) and
returns the package, or None when they have not been built.  Only tests,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py`` use it.

``load(fftw=path)`` imports the build in ``oracle/_ref_fftw`` instead, whose
FFT module leaves the FFTW symbols to the system library at ``path`` (loaded
first, with global symbol visibility): the reference on real FFTW, where a
machine has it.  One process uses one of the two builds.
"""
from __future__ import annotations

import ctypes
import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "_ref")
REF_FFTW = os.path.join(HERE, "_ref_fftw")


def load(fftw=None):
    root = REF
    if fftw:
        root = REF_FFTW
        if not os.path.isdir(os.path.join(root, "janus")):
            return None
        try:
            ctypes.CDLL(fftw, mode=ctypes.RTLD_GLOBAL)
        except OSError:
            return None
    if not os.path.isdir(os.path.join(root, "janus")):
        return None
    if root not in sys.path:
        sys.path.insert(0, root)
    try:
        import janus.fft.serial  # noqa: F401
        import janus.green  # noqa: F401
        import janus.material.elastic.linear.isotropic  # noqa: F401
        import janus.operators  # noqa: F401
    except Exception:
        return None
    import janus
    if "oracle" not in (getattr(janus, "__file__", "") or ""):
        return None
    return janus
