"""Batched mixed-precision solves of cells of uneven sizes in one CUDA graph
per outer step, against the same problems solved one by one (MixedScheme)
and against the plain FP64 scheme."""
import numpy as np
import pytest
import torch

import janus_b200.material.elastic.linear.isotropic as material
from janus_b200 import microstructures as micro
from janus_b200 import operators as ops
from janus_b200.batch import BatchedMixedScheme
from janus_b200.green import filtered, truncated
from janus_b200.solvers import BasicScheme, MixedScheme
from oracle import janus_oracle as O

FACTORY = {"truncated": truncated, "filtered": filtered}


def _operators(p, variant):
    pars = [O.delta_c(g, nu, p["mu0"], p["nu0"], 2) for g, nu in zip(p["mu"], p["nu"])]
    tens = [ops.isotropic_4(s, d, 2) for s, d in pars]
    loc = ops.BlockDiagonalOperator2D.from_phases(p["phase"], tens)
    green = FACTORY[variant](material.create(p["mu0"], p["nu0"], 2).green_operator(),
                             p["phase"].shape, 1.0)
    return green, loc


def _problems(seed, count=6):
    probs = micro.batch_2d_problems(count, seed=seed, sizes=(64, 96, 128, 192, 256))
    for p in probs:  # keep the test short: contrasts up to 50
        p["mu"][1] = min(p["mu"][1], 50.0)
        k = p["mu"] / (1 - 2 * p["nu"])
        p["mu0"] = 0.5 * (p["mu"][0] + p["mu"][1])
        k0 = 0.5 * (k.min() + k.max())
        p["nu0"] = (k0 - p["mu0"]) / (2 * k0)
    return probs


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
def test_batch_matches_one_by_one(variant):
    probs = _problems(1)
    ops_ = [_operators(p, variant) for p in probs]
    E = [np.eye(3) for _ in probs]
    batch = BatchedMixedScheme([(g, l, 3) for g, l in ops_], inner=20, branches=4)
    res = batch.run(E, tol=1e-8, max_outer=2000)
    assert batch.graph_launches == 1   # the whole run in one persistent graph launch
    step = BatchedMixedScheme([(g, l, 3) for g, l in ops_], inner=20, branches=4,
                              persistent=False)
    res_step = step.run(E, tol=1e-8, max_outer=2000)
    assert step.graph_launches == max(r.outer_iterations for r in res) - 1
    for r, q in zip(res, res_step):
        assert torch.equal(r.eps, q.eps) and np.array_equal(r.residuals, q.residuals)
        assert list(r.status) == list(q.status)
    for (g, l), r in zip(ops_, res):
        one = MixedScheme(g, l, 3, inner=20).run(np.eye(3), tol=1e-8, max_outer=2000)
        assert r.outer_iterations == one.outer_iterations
        assert r.fp32_iterations == one.fp32_iterations
        assert np.array_equal(r.residuals, one.residuals)
        assert torch.equal(r.eps, one.eps)
        assert np.array_equal(r.mean_tau, one.mean_tau)
        assert r.residuals[-1].max() <= 1e-8


@pytest.mark.gpu
def test_batch_effective_stiffness_matches_fp64():
    probs = _problems(2, count=4)
    ops_ = [_operators(p, "truncated") for p in probs]
    batch = BatchedMixedScheme([(g, l, 3) for g, l in ops_], inner=20)
    res = batch.run([np.eye(3)] * len(probs), tol=1e-10, max_outer=5000)
    for p, (g, l), r in zip(probs, ops_, res):
        ref = BasicScheme(g, l, 3).run(np.eye(3), 100000, tol=1e-10)
        mat0 = material.create(p["mu0"], p["nu0"], 2)
        c_ref = ref.mean_stress(mat0, np.eye(3))
        c_mix = r.mean_stress(mat0, np.eye(3))
        assert np.abs(c_mix - c_ref).max() <= 1e-7 * np.abs(c_ref).max()


@pytest.mark.gpu
def test_batch_reuses_graph_until_a_problem_leaves():
    probs = _problems(3, count=3)
    ops_ = [_operators(p, "truncated") for p in probs]
    batch = BatchedMixedScheme([(g, l, 3) for g, l in ops_], inner=10, branches=2)
    res = batch.run([np.eye(3)] * 3, tol=1e-6, max_outer=3)
    # stopped by max_outer: every problem made 3 residual evaluations
    assert [r.outer_iterations for r in res] == [3, 3, 3] or \
        all(r.residuals[-1].max() <= 1e-6 or r.outer_iterations == 3 for r in res)
    assert batch.graph_launches <= 2
    with pytest.raises(ValueError):
        batch.run([np.eye(3)] * 2, tol=1e-6)


@pytest.mark.gpu
def test_batch_runs_again_on_new_fields():
    """A second run with new strain fields (and another inner count) must not
    reuse a graph captured for the first run's fields."""
    probs = _problems(4, count=3)
    ops_ = [_operators(p, "truncated") for p in probs]
    batch = BatchedMixedScheme([(g, l, 3) for g, l in ops_], inner=10, branches=3)
    first = batch.run([np.eye(3)] * 3, tol=1e-8, max_outer=500)
    keep = [r.eps.clone() for r in first]
    for r in first:
        r.eps.fill_(float("nan"))
    second = batch.run([np.eye(3)] * 3, tol=1e-8, max_outer=500)
    for k, r in zip(keep, second):
        assert torch.equal(k, r.eps)
    third = batch.run([np.eye(3)] * 3, tol=1e-8, max_outer=500, inner=15)
    for (g, l), r in zip(ops_, third):
        one = MixedScheme(g, l, 3, inner=15).run(np.eye(3), tol=1e-8, max_outer=500)
        assert torch.equal(one.eps, r.eps)


@pytest.mark.gpu
def test_batch_bicgstab_matches_one_by_one():
    probs = _problems(5, count=4)
    ops_ = [_operators(p, "filtered") for p in probs]
    batch = BatchedMixedScheme([(g, l, 3) for g, l in ops_], inner=15, branches=2,
                               method="bicgstab")
    res = batch.run([np.eye(3)] * 4, tol=1e-9, max_outer=200)
    for (g, l), r in zip(ops_, res):
        # the batch graph runs a fixed count per correction
        one = MixedScheme(g, l, 3, inner=15, method="bicgstab_fixed").run(
            np.eye(3), tol=1e-9, max_outer=200)
        assert r.outer_iterations == one.outer_iterations
        assert r.fp32_iterations == one.fp32_iterations
        assert torch.equal(r.eps, one.eps)
        assert r.residuals[-1].max() <= 1e-9


@pytest.mark.gpu
def test_batch_config3_range_long_axes():
    """The batched workload's own range: grids of 384 to 1024 points a side
    (the long-axis Green pass), contrasts up to 1000, 3 load cases, BiCGSTAB
    corrections: bitwise equal to the same cells solved one by one, one
    graph launch, and effective stiffness within 1e-7 of FP64 GMRES on the
    FP64 equation."""
    from janus_b200.solvers import GMRES
    probs = micro.batch_2d_problems(4, seed=11, sizes=(384, 512, 768, 1024))
    probs[0]["mu"][1] = 1000.0          # the top of the contrast range
    for p in probs:
        k = p["mu"] / (1 - 2 * p["nu"])
        p["mu0"] = 0.5 * (p["mu"][0] + p["mu"][1])
        k0 = 0.5 * (k.min() + k.max())
        p["nu0"] = (k0 - p["mu0"]) / (2 * k0)
    ops_ = [_operators(p, "filtered") for p in probs]
    tol = 1e-9
    batch = BatchedMixedScheme([(g, l, 3) for g, l in ops_], inner=25, method="bicgstab")
    res = batch.run([np.eye(3)] * len(probs), tol=tol, max_outer=100)
    assert batch.graph_launches == 1
    for p, (g, l), r in zip(probs, ops_, res):
        assert r.converged and r.residuals[-1].max() <= tol
        one = MixedScheme(g, l, 3, inner=25, method="bicgstab_fixed").run(
            np.eye(3), tol=tol, max_outer=100)
        assert r.outer_iterations == one.outer_iterations
        assert torch.equal(r.eps, one.eps)
        ref = GMRES(g, l, nload=3, restart=20).run(np.eye(3), tol=1e-11, max_iter=20000)
        assert ref.converged
        mat0 = material.create(p["mu0"], p["nu0"], 2)
        c_ref = ref.mean_stress(mat0, np.eye(3))
        c_mix = r.mean_stress(mat0, np.eye(3))
        assert np.abs(c_mix - c_ref).max() <= 1e-7 * np.abs(c_ref).max()
