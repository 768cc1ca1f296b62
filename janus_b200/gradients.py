"""Gradients of mean stresses (effective moduli) with respect to a per-voxel
shear-modulus field mu(x), through the adjoint of the Lippmann-Schwinger
equation.  The reference has no derivatives; this module builds on its
basic scheme (sphinx/tutorials/square_basic/square_basic.py:83-97) and its
mean-stress post-processing (square_basic.py:95-97).

For load case j with macroscopic strain E_j the strain field solves

    (I + Gamma0 dC) eps_j = E_j,        dC = C(x) - C0,

and the mean stress is S_j = C0:E_j + <dC:eps_j>.  For a cotangent G of S
(one row per load case), J = sum_j G_j . S_j has the per-voxel derivative

    dJ/dtheta(x) = (1/N) sum_j zeta_j(x) . dC/dtheta(x) . eps_j(x),
    (I + Gamma0 dC) zeta_j = G_j,

because Gamma0 is self-adjoint: the adjoint field zeta_j is the solution of
the same equation with the cotangent row as the macroscopic strain (the
"transposed right-hand side").  With C = dim k J + 2 mu K (isotropic, nu
fixed), dC/dmu = dim dk/dmu J + 2 K, and the contraction kernel
(``jb_local_gradient``) returns the J and K parts per voxel.  C0 is a
numerical parameter of the scheme (the converged fields do not depend on
it), so it is held fixed.

The adjoint needs only the converged strain fields, not the iterates, so
the forward pass keeps one FP64 field set per microstructure; with
``keep_strain=False`` it keeps nothing and the backward pass solves the
forward problem again (the memory checkpoint for large 3D batches).
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass, field
from typing import Optional

import numpy as np
import torch

from . import _arrays as A
from . import _lib
from .green import filtered, truncated, willot2015
from .material.elastic.linear import isotropic as material
from .operators import LocalPhaseOperator
from .solvers import BasicScheme, MixedScheme

_FACTORY = {"truncated": truncated, "filtered": filtered, "willot": willot2015}


def bulk_factor(nu, dim):
    """k / mu at fixed Poisson ratio: plane strain 1/(1-2nu) in 2D,
    2(1+nu)/(3(1-2nu)) in 3D (isotropic.pyx:74-77)."""
    if dim == 2:
        return 1.0 / (1.0 - 2.0 * nu)
    return 2.0 / 3.0 * (1.0 + nu) / (1.0 - 2.0 * nu)


@dataclass
class StiffnessFieldProblem:
    """A periodic cell whose shear modulus varies per voxel at a uniform
    Poisson ratio ``nu``, loaded by the rows of ``avg_eps``.

    mu0, nu0: reference medium (default: mid-range of the field, nu).
    variant: "truncated", "filtered" or "willot" Green operator; h: voxel size.
    mixed: FP32 bulk iterations with FP64 defect correction (else plain
    FP64), the correction solved by ``inner_method`` ("bicgstab": ``inner``
    BiCGSTAB iterations; "basic": ``inner - 1`` basic iterations); tol:
    relative residual of the basic scheme (both paths stop on it).
    """
    nu: float = 0.3
    avg_eps: Optional[np.ndarray] = None
    mu0: Optional[float] = None
    nu0: Optional[float] = None
    variant: str = "truncated"
    h: float = 1.0
    tol: float = 1e-8
    max_iter: int = 20000
    mixed: bool = True
    inner: int = 25
    inner_method: str = "bicgstab"
    keep_strain: bool = True
    stats: list = field(default_factory=list)   # per solve: (kind, iterations, residual)

    def macro(self, dim):
        s = 3 if dim == 2 else 6
        E = np.eye(s) if self.avg_eps is None else np.asarray(self.avg_eps, dtype=np.float64)
        return np.atleast_2d(E).reshape(-1, s)


class _Cell:
    """The operators of one microstructure: reference medium, Green
    operator and the dC field."""

    def __init__(self, mu, prob):
        self.shape = tuple(mu.shape)
        self.dim = len(self.shape)
        if self.dim not in (2, 3):
            raise ValueError("mu must be a 2D or 3D field")
        mu64 = mu.detach().to(torch.float64)
        lo, hi = float(mu64.min()), float(mu64.max())
        if lo <= 0.0:
            raise ValueError("mu must be > 0")
        self.mu0 = 0.5 * (lo + hi) if prob.mu0 is None else float(prob.mu0)
        self.nu0 = prob.nu if prob.nu0 is None else float(prob.nu0)
        self.mat0 = material.create(self.mu0, self.nu0, self.dim)
        fac = bulk_factor(prob.nu, self.dim)
        self.dsph_dmu = self.dim * fac           # d(dim k)/d mu
        sph = self.dim * (fac * mu64 - self.mat0.k)
        dev = 2.0 * (mu64 - self.mu0)
        self.local = LocalPhaseOperator(self.dim, self.shape, None, sph.flatten(),
                                        dev.flatten(), torch.float64)
        if prob.variant not in _FACTORY:
            raise ValueError("variant must be 'truncated', 'filtered' or 'willot'")
        self.green = _FACTORY[prob.variant](self.mat0.green_operator(), self.shape, prob.h)
        self.prob = prob

    def solve(self, E, kind):
        """Strain fields (nload, *grid, s) for the rows of E (FP64)."""
        prob = self.prob
        if prob.mixed:
            res = MixedScheme(self.green, self.local, E.shape[0], prob.inner,
                              method=prob.inner_method).run(
                E, tol=prob.tol, max_outer=max(1, prob.max_iter // max(prob.inner, 1)))
            its = res.fp32_iterations + res.outer_iterations
        else:
            res = BasicScheme(self.green, self.local, E.shape[0]).run(E, prob.max_iter,
                                                                     tol=prob.tol)
            its = res.iterations
        last = float(res.residuals[-1].max()) if len(res.residuals) else float("nan")
        prob.stats.append((kind, its, last))
        return res


def _gradient(cell, eps, zeta):
    """dJ/dmu per voxel from the strain and adjoint-strain fields."""
    nload = zeta.shape[0]
    nvox = int(np.prod(cell.shape))
    out = torch.empty((nvox, 2), dtype=torch.float64, device=A.device())
    _lib.check(_lib.lib().jb_local_gradient(
        cell.dim, A.jb_dtype(torch.float64), nvox, nload, ctypes.c_void_p(eps.data_ptr()),
        ctypes.c_void_p(zeta.data_ptr()), 1.0 / nvox, ctypes.c_void_p(out.data_ptr()),
        ctypes.c_void_p(A.stream_handle())))
    g = out[:, 0] * cell.dsph_dmu + out[:, 1] * 2.0
    return g.reshape(cell.shape)


class MeanStress(torch.autograd.Function):
    """mu (grid, or batch x grid when ``batched``; CUDA) -> mean stresses
    (nload, s) per microstructure, differentiable with respect to mu by the
    adjoint."""

    @staticmethod
    def forward(ctx, mu, prob, batched):
        if mu.device.type != "cuda":
            raise ValueError("mu must be a CUDA tensor")
        mus = mu if batched else mu.unsqueeze(0)
        outs, cells, strains = [], [], []
        for b in range(mus.shape[0]):
            cell = _Cell(mus[b], prob)
            E = prob.macro(cell.dim)
            res = cell.solve(E, "forward")
            outs.append(torch.from_numpy(res.mean_stress(cell.mat0, E)))
            cells.append(cell)
            strains.append(res.eps if prob.keep_strain else None)
        ctx.prob = prob
        ctx.cells = cells
        ctx.strains = strains
        ctx.batched = batched
        out = torch.stack(outs).to(mu.device)
        return out if batched else out[0]

    @staticmethod
    def backward(ctx, grad_out):
        prob = ctx.prob
        g = grad_out if ctx.batched else grad_out.unsqueeze(0)
        g = g.detach().to(torch.float64).cpu().numpy()
        grads = []
        for b, cell in enumerate(ctx.cells):
            E = prob.macro(cell.dim)
            Gb = g[b]
            rows = [j for j in range(Gb.shape[0]) if np.any(Gb[j] != 0.0)]
            if not rows:
                grads.append(torch.zeros(cell.shape, dtype=torch.float64, device=A.device()))
                continue
            eps = ctx.strains[b]
            if eps is None:
                eps = cell.solve(E, "recompute").eps
            zeta = cell.solve(np.ascontiguousarray(Gb[rows]), "adjoint").eps
            eps_sel = eps[rows].contiguous() if len(rows) < eps.shape[0] else eps
            grads.append(_gradient(cell, eps_sel, zeta))
        out = torch.stack(grads)
        return (out if ctx.batched else out[0]), None, None


def mean_stress(mu, prob=None, batched=False):
    """Mean stresses of the cell with shear-modulus field ``mu`` (a CUDA
    tensor of the grid shape; batch x grid with ``batched``), one row per
    load case of ``prob.avg_eps`` (default: the unit Mandel load cases);
    differentiable with respect to ``mu``."""
    prob = StiffnessFieldProblem() if prob is None else prob
    return MeanStress.apply(mu, prob, bool(batched))


def effective_shear_modulus(mu, prob=None, batched=False):
    """C_1212 = <sigma_xy>/(2 eps_xy) under the xy unit load (Mandel: the
    last component, sigma = sqrt(2) sigma_xy, eps = sqrt(2) eps_xy), as the
    tutorial's post-processing (square_basic.py:95-97); differentiable with
    respect to ``mu``."""
    prob = StiffnessFieldProblem() if prob is None else prob
    dim = mu.dim() - (1 if batched else 0)
    s = 3 if dim == 2 else 6
    E = np.zeros((1, s))
    E[0, -1] = 1.0
    p = StiffnessFieldProblem(**{**prob.__dict__, "avg_eps": E})
    p.stats = prob.stats
    S = MeanStress.apply(mu, p, bool(batched))
    return 0.5 * S[..., 0, -1]
