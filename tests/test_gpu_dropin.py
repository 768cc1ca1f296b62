"""Drop-in use: the reference's own tutorial script, unmodified, on janus_b200.

``install_as_janus()`` aliases the ``janus`` modules to janus_b200; the
tutorial sphinx/tutorials/square_basic/square_basic.py then runs as its own
``__main__`` (its Example class, its 400-iteration numpy loop at lines 83-92
and its post-processing at 94-97) with matplotlib replaced by a stub that
draws nothing.  The printed C_1212 must equal the published value
1.41903971282 (square_basic.rst:227) to 5e-12.

The script is read from the reference checkout named by $JANUS_REFERENCE;
the test skips where there is none.  The planner-flag test needs no
reference."""
import contextlib
import io
import os
import runpy
import sys
import types

import numpy as np
import pytest

import janus_b200.material.elastic.linear.isotropic as material
from janus_b200 import autotune
from janus_b200.fft import serial as fft
from janus_b200.green import truncated
from oracle import janus_oracle as O


def _tutorial_path():
    root = os.environ.get("JANUS_REFERENCE")
    if not root:
        return None
    p = os.path.join(root, "sphinx", "tutorials", "square_basic", "square_basic.py")
    return p if os.path.exists(p) else None


class _Stub:
    """Figure / axes stand-in: every method accepts anything and does nothing."""

    def get_size_inches(self):
        return 6.4, 4.8

    def __getattr__(self, name):
        return lambda *a, **k: None


def _pyplot_stub():
    plt = types.ModuleType("matplotlib.pyplot")

    def subplots(nrows=1, ncols=1, **kw):
        n = nrows * ncols
        return _Stub(), (_Stub() if n == 1 else [_Stub() for _ in range(n)])
    plt.subplots = subplots
    mpl = types.ModuleType("matplotlib")
    mpl.pyplot = plt
    return mpl, plt


@pytest.mark.gpu
def test_reference_tutorial_runs_unmodified(monkeypatch, tmp_path):
    path = _tutorial_path()
    if path is None:
        pytest.skip("no reference checkout ($JANUS_REFERENCE) to read the tutorial from")
    from janus_b200.compat import install_as_janus
    saved = {k: v for k, v in sys.modules.items() if k == "janus" or k.startswith("janus.")}
    for k in saved:
        del sys.modules[k]
    mpl, plt = _pyplot_stub()
    monkeypatch.setitem(sys.modules, "matplotlib", mpl)
    monkeypatch.setitem(sys.modules, "matplotlib.pyplot", plt)
    monkeypatch.chdir(tmp_path)
    try:
        install_as_janus()
        out = io.StringIO()
        with contextlib.redirect_stdout(out):
            runpy.run_path(path, run_name="__main__")
    finally:
        for k in [k for k in sys.modules if k == "janus" or k.startswith("janus.")]:
            del sys.modules[k]
        sys.modules.update(saved)
    c1212 = float(out.getvalue().split()[-1])
    assert abs(c1212 - 1.41903971282) < 5e-12, c1212


@pytest.mark.gpu
def test_patient_planning_runs_the_autotuner_and_measure_reuses_it(monkeypatch, tmp_path):
    """FFTW_PATIENT on the transform: the Green operator's first apply times
    the column schedules and caches the choice; FFTW_MEASURE on a second
    operator of the grid picks the cached schedule without timing;
    FFTW_ESTIMATE keeps the built-in rule.  Every schedule gives the oracle's
    result."""
    monkeypatch.setenv("JB_TUNE_CACHE", str(tmp_path / "tune.json"))
    shape = (32, 24, 20)
    rng = np.random.default_rng(1)
    x = rng.normal(size=shape + (6,))
    ref = O.green_apply(x, 0.75, 0.3, 1.0, "truncated")
    mat = material.create(0.75, 0.3, 3)
    g1 = truncated(mat.green_operator(), shape, 1.0,
                   transform=fft.create_real(shape, flags=fft.FFTW_PATIENT))
    y1 = np.asarray(g1.apply(x))
    assert os.path.exists(tmp_path / "tune.json")
    tuned = autotune.get_tuning(g1)
    g2 = truncated(mat.green_operator(), shape, 1.0,
                   transform=fft.create_real(shape, flags=fft.FFTW_MEASURE))
    calls = []
    monkeypatch.setattr(autotune, "_time_passes", lambda *a, **k: calls.append(1))
    y2 = np.asarray(g2.apply(x))
    assert calls == [] and autotune.get_tuning(g2)[:6] == tuned[:6]
    g3 = truncated(mat.green_operator(), shape, 1.0,
                   transform=fft.create_real(shape, flags=fft.FFTW_ESTIMATE))
    y3 = np.asarray(g3.apply(x))
    assert autotune.get_tuning(g3)[:6] == [0, 0, 1, 0, 0, 1]
    for y in (y1, y2, y3):
        np.testing.assert_allclose(y, ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
