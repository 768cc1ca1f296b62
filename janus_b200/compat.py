"""Drop-in aliasing: make ``import janus.<module>`` resolve to janus_b200.

    import janus_b200.compat
    janus_b200.compat.install_as_janus()
    import janus.green as green          # -> janus_b200.green

Registers the reference's module paths (janus, janus.fft, janus.fft.serial,
janus.green, janus.operators, janus.material.elastic.linear.isotropic) in
``sys.modules``.  Refuses to replace an already-imported ``janus`` package.
"""
from __future__ import annotations

import importlib
import sys

_MODULES = {
    "janus": "janus_b200",
    "janus.fft": "janus_b200.fft",
    "janus.fft.serial": "janus_b200.fft.serial",
    "janus.green": "janus_b200.green",
    "janus.operators": "janus_b200.operators",
    "janus.material": "janus_b200.material",
    "janus.material.elastic": "janus_b200.material.elastic",
    "janus.material.elastic.linear": "janus_b200.material.elastic.linear",
    "janus.material.elastic.linear.isotropic": "janus_b200.material.elastic.linear.isotropic",
}


def install_as_janus(force: bool = False) -> None:
    existing = sys.modules.get("janus")
    if existing is not None and not force and not getattr(existing, "__name__", "").startswith(
            "janus_b200"):
        if getattr(existing, "__file__", None) and "janus_b200" not in existing.__file__:
            raise RuntimeError("a different 'janus' package is already imported")
    for alias, real in _MODULES.items():
        sys.modules[alias] = importlib.import_module(real)
