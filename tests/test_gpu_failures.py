"""Failure reporting of the solvers and the pass kernels, in the forms that
fault no GPU: non-finite and diverging load cases are made on the host (a
NaN in one load case's initial strain field or in the phase table, a
reference medium that makes the basic scheme diverge; a NaN macroscopic
strain is rejected before any work as an invalid argument), and a
timed-out copy wait is made by
cutting the first bounded wait to no poll at all, after which every kernel
drains its own copy at the full limit and returns.

No counterpart in the reference, whose tutorial loop only records the
residuals (sphinx/tutorials/square_basic/square_basic.py:88-92)."""
import numpy as np
import pytest
import torch

import janus_b200.material.elastic.linear.isotropic as material
from janus_b200 import _lib
from janus_b200 import microstructures as micro
from janus_b200 import operators as ops
from janus_b200.batch import BatchedMixedScheme
from janus_b200.green import filtered, truncated
from janus_b200.solvers import GMRES, BasicScheme, MixedScheme
from oracle import janus_oracle as O

CONVERGED, MAX_ITER, NON_FINITE, DIVERGING = 0, 1, 2, 3


def _problem(phase, mats, g0, nu0, variant="truncated", nan_phase=None):
    dim = phase.ndim
    pars = [list(O.delta_c(g, nu, g0, nu0, dim)) for g, nu in mats]
    if nan_phase is not None:
        pars[nan_phase][1] = float("nan")
    tens = [ops.isotropic_4(s, d, dim) for s, d in pars]
    cls = ops.BlockDiagonalOperator2D if dim == 2 else ops.BlockDiagonalOperator3D
    loc = cls.from_phases(phase, tens)
    factory = truncated if variant == "truncated" else filtered
    green = factory(material.create(g0, nu0, dim).green_operator(), phase.shape, 1.0)
    return loc, green


def _nan_start(shape, E):
    """initial fields: E everywhere, load case 1 poisoned at one voxel"""
    eps = torch.empty(shape, dtype=torch.float64, device="cuda")
    eps[...] = torch.from_numpy(E).cuda().view((E.shape[0],) + (1,) * (len(shape) - 2) +
                                                (E.shape[1],))
    eps[(1,) + (0,) * (len(shape) - 1)] = float("nan")
    return eps


@pytest.mark.gpu
def test_basic_scheme_nan_load_case_stops_at_once():
    phase = micro.square_inclusion(64, side=32)
    loc, green = _problem(phase, [(1.0, 0.3), (10.0, 0.3)], 5.5, 0.3)
    E = np.array([[0.0, 0.0, 1.0], [1.0, 0.0, 0.0]])
    s = BasicScheme(green, loc, nload=2)
    with pytest.raises(ValueError, match="nonzero"):
        s.run(np.array([[0.0, 0.0, 1.0], [np.nan, 0.0, 0.0]]), 10)
    r = s.run(E, 500, tol=1e-8, eps=_nan_start(s.field_shape, E), init=False)
    assert list(r.status) == [CONVERGED, NON_FINITE]
    assert r.status_names == ["converged", "non_finite"]
    assert not r.converged
    assert np.isnan(r.residuals[0, 1])
    assert r.residuals[-1, 0] <= 1e-8


@pytest.mark.gpu
def test_basic_scheme_max_iter_and_converged():
    phase = micro.square_inclusion(64, side=32)
    loc, green = _problem(phase, [(1.0, 0.3), (10.0, 0.3)], 5.5, 0.3)
    E = np.array([0.0, 0.0, 1.0])
    r = BasicScheme(green, loc).run(E, 3, tol=1e-8)
    assert list(r.status) == [MAX_ITER] and r.iterations == 3
    r = BasicScheme(green, loc).run(E, 1000, tol=1e-8)
    assert list(r.status) == [CONVERGED] and r.converged


@pytest.mark.gpu
def test_basic_scheme_diverging_reference_medium():
    """mu_0 far below the inclusion's modulus: the basic scheme's iteration
    matrix has spectral radius about 9, the residual grows geometrically and
    the load case stops as diverging long before max_iter."""
    phase = micro.square_inclusion(64, side=32)
    loc, green = _problem(phase, [(1.0, 0.3), (100.0, 0.3)], 10.0, 0.3)
    r = BasicScheme(green, loc).run(np.array([0.0, 0.0, 1.0]), 500, tol=1e-10)
    assert list(r.status) == [DIVERGING]
    assert r.iterations < 50
    assert r.residuals[-1, 0] > 1e4 * r.residuals[:, 0].min()


@pytest.mark.gpu
def test_mixed_scheme_statuses():
    phase, _ = micro.random_spheres(16, radius=3, volume_fraction=0.2, seed=4)
    loc, green = _problem(phase, [(1.0, 0.3), (10.0, 0.3)], 5.5, 0.3, "filtered")
    E = np.zeros((2, 6))
    E[0, 0] = 1.0
    E[1, 2] = 1.0
    m = MixedScheme(green, loc, nload=2, inner=10)
    r = m.run(E, tol=1e-10, max_outer=100, eps=_nan_start(m.field_shape, E))
    assert list(r.status) == [CONVERGED, NON_FINITE]
    # diverging: the FP64 residual of the basic scheme grows outer step by outer step
    loc, green = _problem(phase, [(1.0, 0.3), (100.0, 0.3)], 10.0, 0.3, "filtered")
    r = MixedScheme(green, loc, nload=1, inner=4).run(np.eye(6)[:1], tol=1e-10,
                                                      max_outer=200)
    assert list(r.status) == [DIVERGING] and r.outer_iterations < 60


@pytest.mark.gpu
def test_gmres_nan_phase_table():
    phase = micro.square_inclusion(32, side=16)
    loc, green = _problem(phase, [(1.0, 0.3), (10.0, 0.3)], 5.5, 0.3, nan_phase=1)
    r = GMRES(green, loc, nload=1, restart=10).run(np.array([0.0, 0.0, 1.0]), tol=1e-10,
                                                    max_iter=100)
    assert list(r.status) == [NON_FINITE]
    loc, green = _problem(phase, [(1.0, 0.3), (10.0, 0.3)], 5.5, 0.3)
    r = GMRES(green, loc, nload=1, restart=10).run(np.array([0.0, 0.0, 1.0]), tol=1e-10,
                                                    max_iter=200)
    assert list(r.status) == [CONVERGED]


@pytest.mark.gpu
def test_batch_statuses_per_problem():
    loc0, g0 = _problem(micro.square_inclusion(32, side=16), [(1.0, 0.3), (10.0, 0.3)], 5.5,
                        0.3)
    loc1, g1 = _problem(micro.square_inclusion(48, side=16), [(1.0, 0.3), (100.0, 0.3)], 10.0,
                        0.3)
    b = BatchedMixedScheme([(g0, loc0, 2), (g1, loc1, 1)], inner=6)
    E0 = np.array([[0.0, 0.0, 1.0], [1.0, 0.0, 0.0]])
    E1 = np.array([[1.0, 0.0, 0.0]])
    e1 = torch.empty(b.schemes[1].field_shape, dtype=torch.float64, device="cuda")
    e1[...] = torch.from_numpy(E1).cuda().view(1, 1, 1, 3)
    out = b.run([E0, E1], tol=1e-9, max_outer=80,
                eps=[_nan_start(b.schemes[0].field_shape, E0), e1])
    assert list(out[0].status) == [CONVERGED, NON_FINITE]
    assert list(out[1].status) == [DIVERGING]


@pytest.mark.gpu
def test_timed_out_copy_wait_is_reported():
    """First bounded wait cut to no poll at all: every kernel that waits on a
    bulk copy gives up at once, drains its copy at the full limit and
    returns; the host sees the fault word at the next synchronisation
    (RuntimeError), and the context stays usable once the limit is
    restored."""
    shape = (64, 64, 64)
    rng = np.random.default_rng(0)
    x = rng.normal(size=shape + (6,))
    g = truncated(material.create(0.75, 0.3, 3).green_operator(), shape, 1.0)
    _lib.device_status()  # clear
    try:
        _lib.set_wait_limit(0)
        with pytest.raises(RuntimeError, match="bounded wait"):
            g.apply(x)
        # a 3D cell: its row and axis-1 passes wait on their bulk copies
        phase, _ = micro.random_spheres(64, radius=8, volume_fraction=0.2, seed=1)
        loc, green = _problem(phase, [(1.0, 0.3), (10.0, 0.3)], 5.5, 0.3)
        with pytest.raises(RuntimeError, match="bounded wait"):
            BasicScheme(green, loc).run(np.eye(6)[:1], 5)
        # a 2D cell on 1024-point rows: the persistent long-row kernels give
        # up at their first wait and let the other row buffers' copies land
        # (three load cases, so every CTA has rows queued behind the first)
        phase2 = (rng.random((300, 1024)) < 0.3).astype(np.uint8)
        loc2, green2 = _problem(phase2, [(1.0, 0.3), (10.0, 0.3)], 5.5, 0.3, "filtered")
        with pytest.raises(RuntimeError, match="bounded wait"):
            BasicScheme(green2, loc2, nload=3).run(np.eye(3), 3)
    finally:
        _lib.set_wait_limit()
        _lib.device_status()
    # the same apply is right again with the default limit
    y = np.asarray(g.apply(x))
    ref = O.green_apply(x, 0.75, 0.3, 1.0, "truncated")
    np.testing.assert_allclose(y, ref, rtol=1e-13, atol=1e-13 * np.abs(ref).max())
    assert _lib.device_status() == 0
