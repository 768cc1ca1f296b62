"""Loader of the reference checker (test infrastructure only).

``load()`` imports the reference's own Cython modules compiled by
``oracle/build_ref.py`` into ``oracle/_ref`` (package name ``janus``) and
returns the package, or None when they have not been built.  Only tests,
``__graft_entry__.smoke()`` and the CPU-baseline legs of ``bench.py`` use it.
"""
from __future__ import annotations

import os
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REF = os.path.join(HERE, "_ref")


def load():
    if not os.path.isdir(os.path.join(REF, "janus")):
        return None
    if REF not in sys.path:
        sys.path.insert(0, REF)
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
