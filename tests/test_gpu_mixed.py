"""Mixed-precision basic scheme (FP32 bulk, FP64 defect correction) against
the FP64 GPU solver and the oracle: same residual definition, effective
stiffness within 1e-7 of the FP64 result."""
import numpy as np
import pytest

import janus_b200.material.elastic.linear.isotropic as material
from janus_b200 import microstructures as micro
from janus_b200 import operators as ops
from janus_b200.green import filtered, truncated
from janus_b200.solvers import BasicScheme, MixedScheme
from oracle import janus_oracle as O

FACTORY = {"truncated": truncated, "filtered": filtered}


def _problem(phase, mats, g0, nu0, variant):
    dim = phase.ndim
    pars = [O.delta_c(g, nu, g0, nu0, dim) for g, nu in mats]
    tens = [ops.isotropic_4(s, d, dim) for s, d in pars]
    cls = ops.BlockDiagonalOperator2D if dim == 2 else ops.BlockDiagonalOperator3D
    loc = cls.from_phases(phase, tens)
    green = FACTORY[variant](material.create(g0, nu0, dim).green_operator(), phase.shape, 1.0)
    return loc, green, pars


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
def test_mixed_matches_fp64_3d(variant):
    phase, _ = micro.random_spheres(32, radius=4, volume_fraction=0.3, seed=3)
    mats = [(1.0, 0.3), (100.0, 0.2)]
    g0, nu0 = 50.5, 0.3
    loc, green, pars = _problem(phase, mats, g0, nu0, variant)
    E = np.eye(6)
    tol = 1e-10
    ref = BasicScheme(green, loc, nload=6).run(E, 5000, tol=tol)
    mix = MixedScheme(green, loc, nload=6, inner=20).run(E, tol=tol, max_outer=500)
    assert mix.residuals[-1].max() <= tol
    mat0 = material.create(g0, nu0, 3)
    c_ref = ref.mean_stress(mat0, E)
    c_mix = mix.mean_stress(mat0, E)
    assert np.abs(c_mix - c_ref).max() <= 1e-7 * np.abs(c_ref).max()
    err = (ref.eps - mix.eps).abs().max().item() / ref.eps.abs().max().item()
    assert err <= 1e-8
    # FP32 does most of the work
    assert mix.fp32_iterations >= 10 * mix.outer_iterations
    # the oracle's effective stiffness for one load case
    eps_o, _, tau_o = O.basic_scheme(phase, [p[0] for p in pars], [p[1] for p in pars], g0,
                                     nu0, E[5], 5000, variant=variant, tol=tol)
    c_o = O.isotropic_apply(E[5], 3 * mat0.k, 2 * mat0.g, 3) + tau_o
    assert np.abs(c_mix[5] - c_o).max() <= 1e-7 * np.abs(c_o).max()


@pytest.mark.gpu
def test_mixed_2d_square():
    phase = micro.square_inclusion(128, side=64)
    loc, green, pars = _problem(phase, [(1.0, 0.3), (100.0, 0.3)], 50.5, 0.3, "truncated")
    E = np.eye(3)
    ref = BasicScheme(green, loc, nload=3).run(E, 5000, tol=1e-10)
    mix = MixedScheme(green, loc, nload=3, inner=10).run(E, tol=1e-10, max_outer=1000)
    mat0 = material.create(50.5, 0.3, 2)
    c_ref = ref.mean_stress(mat0, E)
    c_mix = mix.mean_stress(mat0, E)
    assert np.abs(c_mix - c_ref).max() <= 1e-7 * np.abs(c_ref).max()
    assert mix.residuals[-1].max() <= 1e-10


@pytest.mark.gpu
def test_mixed_rejects_fp32_operators():
    phase = micro.square_inclusion(32, side=16)
    pars = [O.delta_c(1.0, 0.3, 5.5, 0.3, 2), O.delta_c(10.0, 0.3, 5.5, 0.3, 2)]
    tens = [ops.isotropic_4(s, d, 2) for s, d in pars]
    loc = ops.BlockDiagonalOperator2D.from_phases(phase, tens, dtype="float32")
    green = truncated(material.create(5.5, 0.3, 2).green_operator(), phase.shape, 1.0,
                      dtype="float32")
    with pytest.raises(ValueError):
        MixedScheme(green, loc)


@pytest.mark.gpu
@pytest.mark.parametrize("variant", ["truncated", "filtered"])
def test_mixed_bicgstab_matches_fp64_3d(variant):
    """Krylov inner solver (BiCGSTAB on the basic scheme's own operator, as
    the reference's examples/square_inclusion_scipy.py uses gmres): same FP64
    residual and stopping test, same effective stiffness, far fewer
    operator applications."""
    phase, _ = micro.random_spheres(32, radius=4, volume_fraction=0.3, seed=3)
    mats = [(1.0, 0.3), (100.0, 0.2)]
    g0, nu0 = 50.5, 0.3
    loc, green, pars = _problem(phase, mats, g0, nu0, variant)
    E = np.eye(6)
    tol = 1e-10
    ref = BasicScheme(green, loc, nload=6).run(E, 5000, tol=tol)
    kr = MixedScheme(green, loc, nload=6, inner=25, method="bicgstab").run(E, tol=tol,
                                                                          max_outer=100)
    assert kr.residuals[-1].max() <= tol
    assert np.isfinite(kr.eps.cpu().numpy()).all()
    mat0 = material.create(g0, nu0, 3)
    c_ref = ref.mean_stress(mat0, E)
    c_kr = kr.mean_stress(mat0, E)
    assert np.abs(c_kr - c_ref).max() <= 1e-7 * np.abs(c_ref).max()
    err = (ref.eps - kr.eps).abs().max().item() / ref.eps.abs().max().item()
    assert err <= 1e-8
    # fp32_iterations counts applications of the operator
    assert kr.fp32_iterations < 0.5 * ref.iterations


@pytest.mark.gpu
def test_mixed_bicgstab_high_contrast_2d():
    phase = micro.square_inclusion(128, side=64)
    loc, green, pars = _problem(phase, [(1.0, 0.3), (1000.0, 0.3)], 500.5, 0.3, "truncated")
    E = np.eye(3)
    ref = BasicScheme(green, loc, nload=3).run(E, 50000, tol=1e-9)
    kr = MixedScheme(green, loc, nload=3, inner=25, method="bicgstab").run(
        E, tol=1e-9, max_outer=200)
    mat0 = material.create(500.5, 0.3, 2)
    c_ref = ref.mean_stress(mat0, E)
    c_kr = kr.mean_stress(mat0, E)
    assert kr.residuals[-1].max() <= 1e-9
    assert np.abs(c_kr - c_ref).max() <= 1e-7 * np.abs(c_ref).max()
    assert kr.fp32_iterations < 0.2 * ref.iterations


@pytest.mark.gpu
def test_mixed_bicgstab_homogeneous_cell_stays_finite():
    """dC constant: the LS solution is E itself, the first residual is zero
    and no Krylov scalar may turn into NaN."""
    phase = np.zeros((32, 32), dtype=np.uint8)
    loc, green, pars = _problem(phase, [(3.0, 0.3)], 5.5, 0.3, "filtered")
    E = np.eye(3)
    r = MixedScheme(green, loc, nload=3, inner=10, method="bicgstab").run(E, tol=1e-12,
                                                                        max_outer=5)
    assert np.isfinite(r.eps.cpu().numpy()).all()
    assert np.abs(r.eps.cpu().numpy() - E.reshape(3, 1, 1, 3)).max() <= 1e-12


@pytest.mark.gpu
@pytest.mark.parametrize("method", ["basic", "bicgstab"])
def test_fp64_inner_control_matches_fp64(method):
    """The same defect correction with FP64 corrections (the precision
    control): converges to the FP64 basic scheme's solution, and with BiCGSTAB
    in a handful of outer steps."""
    import torch
    phase, _ = micro.random_spheres(32, radius=4, volume_fraction=0.3, seed=5)
    mats = [(1.0, 0.3), (100.0, 0.2)]
    g0, nu0 = 50.5, 0.3
    loc, green, pars = _problem(phase, mats, g0, nu0, "truncated")
    E = np.eye(6)[[0, 5]]
    tol = 1e-10
    ref = BasicScheme(green, loc, nload=2).run(E, 5000, tol=tol)
    ctl = MixedScheme(green, loc, nload=2, inner=20, method=method,
                      inner_dtype=torch.float64).run(E, tol=tol, max_outer=500)
    assert ctl.converged and ctl.residuals[-1].max() <= tol
    mat0 = material.create(g0, nu0, 3)
    c_ref = ref.mean_stress(mat0, E)
    c_ctl = ctl.mean_stress(mat0, E)
    assert np.abs(c_ctl - c_ref).max() <= 1e-8 * np.abs(c_ref).max()
    if method == "bicgstab":
        assert ctl.outer_iterations <= 10
