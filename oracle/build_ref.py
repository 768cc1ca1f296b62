"""Build the reference's own serial path as a checker (test infrastructure).

This script compiles the reference's Cython modules, unchanged, from where
they lie in the reference tree, against the project-written FFTW-compatible
FFT in ``oracle/fftw_shim`` (libfftw3 is not installed in this image).  All
outputs go to ``oracle/_ref/`` (git-ignored; the built ``.so`` files travel
with the repository snapshot so the checker also runs where the reference
tree is absent):

    oracle/_ref/janus/utils/checkarray*.so          janus/utils/checkarray.pyx
    oracle/_ref/janus/operators*.so                 janus/operators.pyx
    oracle/_ref/janus/material/elastic/linear/isotropic*.so
    oracle/_ref/janus/fft/serial/_serial_fft*.so    janus/fft/serial/_serial_fft.pyx
    oracle/_ref/janus/green*.so                     janus/green.pyx

A second tree, ``oracle/_ref_fftw/``, holds the same modules with the FFT
module linked against nothing: its FFTW symbols resolve at import time to a
system libfftw3 loaded first (``oracle/reference.py``, ``load(fftw=...)``),
for machines that have FFTW.

The package ``__init__.py`` files under ``oracle/_ref/janus`` are written by
this script (minimal re-exports), not copied.  Nothing in the janus_b200
product imports ``oracle/``; only tests, ``__graft_entry__.smoke()`` and the
CPU-baseline legs of ``bench.py`` use it, as the checker.

Usage: ``python oracle/build_ref.py [--reference PATH] [--if-present]``
(default PATH: ``$JANUS_REFERENCE``, else the recipe's checkout location).
Exits non-zero with a message if Cython or the reference tree is unavailable,
unless ``--if-present`` is given (then a missing tree is a no-op).
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
import sysconfig

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_ref")
OUT_FFTW = os.path.join(HERE, "_ref_fftw")
SHIM = os.path.join(HERE, "fftw_shim")

MODULES = [
    "janus/utils/checkarray",
    "janus/operators",
    "janus/material/elastic/linear/isotropic",
    "janus/fft/serial/_serial_fft",
    "janus/green",
]

INIT_FILES = {
    "janus/__init__.py": "",
    "janus/utils/__init__.py": "",
    "janus/material/__init__.py": "",
    "janus/material/elastic/__init__.py": "",
    "janus/material/elastic/linear/__init__.py": "",
    "janus/fft/__init__.py": (
        "from .serial._serial_fft import (FFTW_ESTIMATE, FFTW_MEASURE, "
        "FFTW_PATIENT, FFTW_EXHAUSTIVE, FFTW_WISDOM_ONLY, FFTW_DESTROY_INPUT, "
        "FFTW_PRESERVE_INPUT, FFTW_UNALIGNED, FFTW_CONSERVE_MEMORY)\n"),
    "janus/fft/serial/__init__.py": "from ._serial_fft import create_real\n",
}


def _run(cmd):
    subprocess.run(cmd, check=True)


def build(reference: str) -> None:
    try:
        from Cython.Build import cythonize
    except ImportError as exc:  # pragma: no cover
        raise SystemExit(f"Cython is required to build the checker: {exc}")
    if not os.path.isdir(os.path.join(reference, "janus")):
        raise SystemExit(f"reference tree not found at {reference}")
    os.makedirs(OUT, exist_ok=True)
    cbuild = os.path.join(OUT, "build")
    os.makedirs(cbuild, exist_ok=True)

    shim_obj = os.path.join(cbuild, "fftw_shim.o")
    _run(["gcc", "-O2", "-fPIC", "-c", os.path.join(SHIM, "fftw_shim.c"),
          "-I", SHIM, "-o", shim_obj])

    cwd = os.getcwd()
    os.chdir(reference)  # module names follow the reference's package tree
    try:
        sources = [m + ".pyx" for m in MODULES]
        cythonize(sources, build_dir=cbuild, include_path=[reference],
                  language_level=3, quiet=True, force=True)
    finally:
        os.chdir(cwd)

    py_inc = sysconfig.get_paths()["include"]
    ext = sysconfig.get_config_var("EXT_SUFFIX")
    for out, shim in ((OUT, True), (OUT_FFTW, False)):
        for mod in MODULES:
            csrc = os.path.join(cbuild, mod + ".c")
            target = os.path.join(out, mod + ext)
            os.makedirs(os.path.dirname(target), exist_ok=True)
            cmd = ["gcc", "-O2", "-fPIC", "-shared", "-fno-strict-aliasing",
                   "-w", "-I", py_inc, "-I", SHIM, csrc, "-o", target]
            if shim and mod.endswith("_serial_fft"):
                cmd[-2:-2] = [shim_obj]
            cmd.append("-lm")
            _run(cmd)
        for rel, text in INIT_FILES.items():
            path = os.path.join(out, rel)
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as f:
                f.write(text)
    shutil.rmtree(cbuild, ignore_errors=True)
    print(f"checker built in {OUT}")


# where the reference tree is read from: $JANUS_REFERENCE, else the
# recipe's default checkout location
DEFAULT_REFERENCE = os.environ.get("JANUS_REFERENCE", "/root/reference")


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--reference", default=DEFAULT_REFERENCE)
    ap.add_argument("--if-present", action="store_true",
                    help="exit 0 with a note when the reference tree is absent")
    args = ap.parse_args(argv)
    if args.if_present and not os.path.isdir(os.path.join(args.reference, "janus")):
        print(f"reference tree not found at {args.reference}: checker not rebuilt")
        return
    build(args.reference)


if __name__ == "__main__":
    main()
