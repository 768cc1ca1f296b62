"""Autotuner for the column-pass tile schedules of a Green operator.

No counterpart in the reference, which leaves planning to FFTW
(``flags=FFTW_MEASURE``, janus/fft/serial/_serial_fft.pyx:20-53).  Here the
FFT radices follow from the axis length (compile-time radix-16/8 tiles for
n = 64, 128, 256; runtime mixed-radix plans otherwise); what is tuned is how
the column passes tile the spectrum: the width of a tile in complex columns,
how many input tiles rotate through shared memory, whether the compile-time
tiles are used (for the Green pass also in place, without a partner tile,
24 columns wide at n = 128 and 12 at n = 256, or the pass whose transforms
and contraction run in registers, n0 = 32 ... 1024), and
whether the Green contraction reads the per-coefficient table of symmetric
Mandel matrices or evaluates the operator on the fly.  Each candidate is timed on the solver step it
will serve (CUDA events around every pass, several steps after a warm-up),
the plain passes (3D axis 1) and the Green pass independently, and the
fastest of each is set on the operator.  Results are cached per GPU model,
grid, precision, variant and load-case count in a JSON file
(``$JB_TUNE_CACHE``, default ``~/.cache/janus_b200/tune.json``).
"""
from __future__ import annotations

import ctypes
import json
import os

import numpy as np
import torch

from . import _lib
from .solvers import BasicScheme

_PLAIN_PASSES = ("cols_fwd_axis1", "cols_inv_axis1")
_GREEN_PASS = "cols_green_axis0"


def get_tuning(green_op):
    """[plain width, plain input tiles, plain compile-time, Green width,
    Green input tiles, Green compile-time, contraction mode]"""
    v = (ctypes.c_int * 7)()
    _lib.check(_lib.lib().jb_green_get_tuning(green_op.handle, v, 7))
    return list(v)


def set_tuning(green_op, values):
    """6 values (schedules) or 7 (with the contraction mode: 0 rule, 1
    table, 2 on the fly)."""
    values = [int(x) for x in values]
    v = (ctypes.c_int * len(values))(*values)
    _lib.check(_lib.lib().jb_green_set_tuning(green_op.handle, v, len(values)))


def candidates(dim, dtype):
    """(plain, green) candidate lists of (width, input tiles, compile-time)."""
    s = 3 if dim == 2 else 6
    plain = [(w, nb, 1) for w in (4, 8, 16) for nb in (2, 3)] + [(8, 2, 0), (8, 3, 0)]
    green = [(w, nb, 1) for w in (s, 2 * s, 3 * s) for nb in (2, 3)] + [(s, 2, 0),
                                                                          (2 * s, 2, 0)]
    # tiles transformed in place: 24 columns at n = 128, 12 at n = 256 (other
    # lengths run these as ordinary compile-time or runtime-plan tiles); the
    # pass whose transforms run in registers (n0 = 32 ... 1024; its tile is
    # fixed; other lengths run the compile-time tiles)
    green += [(24, 2, 2), (12, 2, 2), (0, 0, 3)]
    return (plain if dim == 3 else []), green


def _cache_path():
    return os.environ.get("JB_TUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "janus_b200",
                                       "tune.json"))


def _key(green_op, nload):
    name = torch.cuda.get_device_name() if torch.cuda.is_available() else "cpu"
    dt = "f64" if green_op.dtype == torch.float64 else "f32"
    return "{}|{}|{}|{}|{}".format(name, "x".join(str(v) for v in green_op.ishape[:-1]), dt,
                                   type(green_op).__name__, int(nload))


def timing_local(green_op):
    """A one-phase local operator with (C - C0) = 0 on the Green operator's
    grid and precision: the pass times of a solver step do not depend on the
    material, so the tuner can time the Green operator alone with it."""
    from .operators import LocalPhaseOperator
    grid = tuple(green_op.ishape[:-1])
    return LocalPhaseOperator(len(grid), grid, np.zeros(grid, dtype=np.uint8), [0.0], [0.0],
                              dtype=green_op.dtype)


def _load_cache(path):
    if os.path.exists(path):
        try:
            with open(path) as f:
                return json.load(f)
        except (OSError, ValueError):
            pass
    return {}


def apply_cached(green_op, nload=1):
    """Set the cached schedule of (green_op, nload) if the cache has one
    (FFTW_MEASURE / FFTW_WISDOM_ONLY planning); True when set."""
    entry = _load_cache(_cache_path()).get(_key(green_op, nload))
    if entry is None:
        return False
    set_tuning(green_op, entry["tuning"])
    return True


def _time_passes(solver, eps, res, steps, warmup):
    for _ in range(warmup):
        solver.step(eps, res)
    solver.timing_begin(steps)
    for _ in range(steps):
        solver.step(eps, res)
    ms, n = solver.timing_end()
    return {k: v / max(n, 1) for k, v in ms.items()}


def tune(green_op, local_op=None, nload=1, steps=5, warmup=2, use_cache=True):
    """Time the candidates on a solver step of (green_op, local_op, nload),
    set the fastest schedules on green_op and return
    {"tuning": [6 values], "plain_ms": ..., "green_ms": ..., "cached": bool}.
    Without local_op the passes are timed with a zero-contrast one."""
    path = _cache_path()
    key = _key(green_op, nload)
    cache = _load_cache(path) if use_cache else {}
    if use_cache and key in cache:
        set_tuning(green_op, cache[key]["tuning"])
        return dict(cache[key], cached=True)
    dim = len(green_op.ishape) - 1
    if local_op is None:
        local_op = timing_local(green_op)
    solver = BasicScheme(green_op, local_op, nload)
    s = green_op.ishape[-1]
    E = np.eye(s)[np.arange(nload) % s]
    solver.set_load(E)
    eps = solver.new_field()
    eps[...] = torch.from_numpy(E).to(eps.dtype).to(eps.device).view(
        (nload,) + (1,) * dim + (s,))
    res = torch.zeros(nload, dtype=torch.float64, device=eps.device)
    plain_c, green_c = candidates(dim, green_op.dtype)
    base = get_tuning(green_op)[:6]
    best_plain, best_green = (base[0:3], float("inf")), (base[3:6] + [0], float("inf"))
    def timed(values):
        """Pass times with the schedule `values`; None where a candidate
        does not fit this grid (the native call rejects its tile)."""
        try:
            set_tuning(green_op, values)
            return _time_passes(solver, eps, res, steps, warmup)
        except ValueError:
            return None
    # plain passes (3D): vary the plain schedule, Green schedule fixed
    for c in plain_c:
        t = timed(list(c) + base[3:6])
        if t is None:
            continue
        ms = sum(t.get(p, 0.0) for p in _PLAIN_PASSES)
        if ms < best_plain[1]:
            best_plain = (list(c), ms)
    for mode in (1, 2):   # table, on the fly
        for c in green_c:
            t = timed(best_plain[0] + list(c) + [mode])
            if t is None:
                continue
            ms = t.get(_GREEN_PASS, float("inf"))
            if ms < best_green[1]:
                best_green = (list(c) + [mode], ms)
    chosen = best_plain[0] + best_green[0]
    set_tuning(green_op, chosen)
    out = {"tuning": chosen, "plain_ms": best_plain[1] if plain_c else None,
           "green_ms": best_green[1]}
    if use_cache:
        cache[key] = out
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as f:
                json.dump(cache, f, indent=1, sort_keys=True)
        except OSError:
            pass
    return dict(out, cached=False)
