"""Generate the golden fixtures used by the parity tests.

Reads the reference's 18 golden ``apply`` files (``tests/data/*.npz`` of the
reference tree: Gamma0 applied to a unit polarization block, produced by an
independent external code, compared by the reference at rtol=ULP,
atol=10*ULP in tests/test_discrete_green_operator.py:178-199) and writes a
compact fixture, ``green_apply_golden.npz``, that travels with the repository:

* the input ``x`` is NOT stored: it is a block of ones on one Mandel
  component, rebuilt from the block size and offsets in the file name and the
  component index stored in the fixture (taken from the file's own ``x``: in
  the two 2D filtered files the component does not follow the name, ``xx``
  holds component 1 and ``yy`` component 0); the script checks that the
  rebuild is exact;
* ``y`` is stored at a seeded sample of voxels (all components), plus three
  full-field checksums (sum, sum of squares, and a seeded +-1-weighted sum).

Usage: ``python tests/golden/make_golden.py [--reference PATH]``.
"""
from __future__ import annotations

import argparse
import glob
import os
import re
import zlib

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "green_apply_golden.npz")
NSAMPLE = 768
COMPONENTS = {2: ["xx", "yy", "xy"], 3: ["xx", "yy", "zz", "yz", "zx", "xy"]}
PATTERN = re.compile(
    r"(truncated|filtered)_green_operator_([0-9x]+)_unit_tau_([a-z]+)_"
    r"([0-9x]+)\+([0-9+]+)\.npz")


def parse(name):
    m = PATTERN.fullmatch(name)
    variant, shape, comp, block, offs = m.groups()
    shape = tuple(int(v) for v in shape.split("x"))
    block = tuple(int(v) for v in block.split("x"))
    offs = tuple(int(v) for v in offs.split("+"))
    return variant, shape, COMPONENTS[len(shape)].index(comp), block, offs


def unit_block(shape, comp, block, offs):
    dim = len(shape)
    x = np.zeros(shape + (3 if dim == 2 else 6,))
    sl = tuple(slice(o, o + b) for o, b in zip(offs, block))
    x[sl + (comp,)] = 1.0
    return x


def checksum_weights(shape, s, seed=20240611):
    rng = np.random.default_rng(seed)
    return rng.choice(np.array([-1.0, 1.0]), size=shape + (s,))


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--reference",
                    default=os.environ.get("JANUS_REFERENCE", "/root/reference"),
                    help="reference checkout (default $JANUS_REFERENCE)")
    args = ap.parse_args(argv)
    files = sorted(glob.glob(os.path.join(args.reference, "tests", "data",
                                          "*_green_operator_*.npz")))
    if len(files) != 18:
        raise SystemExit(f"expected 18 golden files, found {len(files)}")
    out = {}
    names = []
    for path in files:
        name = os.path.basename(path)
        variant, shape, _, block, offs = parse(name)
        with np.load(path) as f:
            x, y = f["x"], f["y"]
        comps = np.unique(np.argwhere(x != 0)[:, -1])
        if comps.size != 1:
            raise SystemExit(f"{name}: expected one loaded component")
        comp = int(comps[0])
        xr = unit_block(shape, comp, block, offs)
        if not np.array_equal(x, xr):
            raise SystemExit(f"unit-block rebuild differs for {name}")
        rng = np.random.default_rng(zlib.crc32(name.encode()))
        nvox = int(np.prod(shape))
        idx = np.sort(rng.choice(nvox, size=NSAMPLE, replace=False))
        ys = y.reshape(nvox, -1)[idx]
        w = checksum_weights(shape, y.shape[-1])
        key = name[:-4]
        names.append(key)
        out[key + "/comp"] = np.array(comp)
        out[key + "/idx"] = idx.astype(np.int64)
        out[key + "/y"] = ys
        out[key + "/checksums"] = np.array(
            [y.sum(), (y * y).sum(), (w * y).sum()])
    out["names"] = np.array(names)
    np.savez_compressed(OUT, **out)
    print(f"wrote {OUT} ({os.path.getsize(OUT)} bytes)")


if __name__ == "__main__":
    main()
