"""The basic fixed-point scheme for the Lippmann-Schwinger equation.

The reference library has no solver function: its tutorial loop
(sphinx/tutorials/square_basic/square_basic.py:83-97) composes the local
operator and the Green operator,

    eps_0 = E,   eps_{k+1} = E - Gamma0[(C - C0):eps_k],
    res_k = ||eps_{k+1} - eps_k|| / (sqrt(N) ||E||),

and post-processes <tau> = mean((C - C0):eps) into the effective stiffness
(square_basic.py:95-97).  ``BasicScheme`` runs exactly that loop on the GPU
for several macroscopic load cases at once, with each iteration as five
(3D) or three (2D) fused passes: the local operator inside the first FFT
pass and the update plus FP64 residual reduction inside the last.
"""
from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np
import torch

from . import _arrays as A
from . import _lib
from .operators import LocalPhaseOperator, _BlockDiagonalOperator


class _Outcome:
    """Per-load-case outcome (``status``: ints, 0 converged, 1 max_iter,
    2 non_finite, 3 diverging; no counterpart in the reference, whose loop
    records residuals only)."""

    @property
    def status_names(self):
        return _lib.status_names(self.status)

    @property
    def converged(self):
        return bool(np.all(self.status == 0))


@dataclass
class SolveResult(_Outcome):
    eps: torch.Tensor          # (nload,) + grid + (s,) on the device
    residuals: np.ndarray      # (iterations, nload)
    iterations: int
    mean_tau: np.ndarray       # (nload, s): grid mean of (C - C0):eps
    status: np.ndarray = None  # (nload,) int32, see _Outcome

    def mean_stress(self, mat0, avg_eps):
        """<sigma> = C0:E + <tau> (square_basic.py:95-96, Mandel form)."""
        return _c0_apply(mat0, np.atleast_2d(avg_eps)) + self.mean_tau


def _c0_apply(mat0, E):
    dim = mat0.dim
    sph, dev = dim * mat0.k, 2 * mat0.g
    tr = (sph - dev) / dim
    out = dev * E
    out[:, :dim] += tr * E[:, :dim].sum(axis=1, keepdims=True)
    return out


class BasicScheme:
    """Basic scheme on `nload` load cases with a Green operator from
    janus_b200.green and a phase-map local operator."""

    def __init__(self, green_op, local_op, nload=1):
        if isinstance(local_op, _BlockDiagonalOperator):
            local = local_op.local
            if local is None:
                raise ValueError("the solver needs isotropic local operators (phase map)")
        elif isinstance(local_op, LocalPhaseOperator):
            local = local_op
        else:
            raise TypeError("local_op must be a BlockDiagonalOperator or LocalPhaseOperator")
        if tuple(local.shape) != tuple(green_op.ishape[:-1]):
            raise ValueError("local and green operators must share the grid")
        self.green_op = green_op
        self.local = local
        self.nload = int(nload)
        self.dtype = green_op.dtype
        if local.dtype != self.dtype:
            raise ValueError("local and green operators must share the dtype")
        self._handle = ctypes.c_void_p()
        _lib.check(_lib.lib().jb_solver_create(green_op.handle, local.handle, self.nload,
                                               ctypes.byref(self._handle)))

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().jb_solver_destroy(h)
            except Exception:
                pass
            self._handle = None

    @property
    def field_shape(self):
        return (self.nload,) + tuple(self.green_op.ishape)

    def _macro(self, avg_eps):
        E = np.ascontiguousarray(np.asarray(avg_eps, dtype=np.float64).reshape(
            self.nload, self.green_op.ishape[-1]))
        return E

    def new_field(self):
        return torch.empty(self.field_shape, dtype=self.dtype, device=A.device())

    def run(self, avg_eps, num_iter, tol=0.0, eps=None, init=None):
        """Iterate until every load case has res <= tol, at most num_iter
        times.  eps (device tensor of field_shape) is updated in place; if
        omitted a new field set to E is used."""
        E = self._macro(avg_eps)
        if eps is None:
            eps = self.new_field()
            init = True if init is None else init
        elif tuple(eps.shape) != self.field_shape or eps.dtype != self.dtype or \
                not eps.is_contiguous() or eps.device.type != "cuda":
            raise ValueError("eps must be a contiguous CUDA tensor of shape {0}".format(
                self.field_shape))
        res = np.zeros((max(int(num_iter), 1), self.nload))
        it = ctypes.c_int(0)
        mean = np.zeros((self.nload, self.green_op.ishape[-1]))
        status = np.zeros(self.nload, dtype=np.int32)
        P = ctypes.POINTER(ctypes.c_double)
        _lib.check(_lib.lib().jb_solver_run(
            self._handle, E.ctypes.data_as(P), ctypes.c_void_p(eps.data_ptr()), int(bool(init)),
            int(num_iter), float(tol), res.ctypes.data_as(P), ctypes.byref(it),
            mean.ctypes.data_as(P), status.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
            ctypes.c_void_p(A.stream_handle())))
        n = it.value
        return SolveResult(eps=eps, residuals=res[:n].copy(), iterations=n, mean_tau=mean,
                           status=status)

    def set_load(self, avg_eps):
        E = self._macro(avg_eps)
        _lib.check(_lib.lib().jb_solver_set_load(
            self._handle, E.ctypes.data_as(ctypes.POINTER(ctypes.c_double))))

    def timing_begin(self, max_steps):
        """Record CUDA events around each pass of the next max_steps steps."""
        _lib.check(_lib.lib().jb_solver_timing_begin(self._handle, int(max_steps)))

    def timing_end(self):
        """{pass name: total device ms} over the recorded steps, and the
        number of steps recorded."""
        ms = (ctypes.c_double * 8)()
        npass = ctypes.c_int(0)
        nsteps = ctypes.c_int(0)
        _lib.check(_lib.lib().jb_solver_timing_end(self._handle, ms, ctypes.byref(npass),
                                                   ctypes.byref(nsteps)))
        names = [_lib.lib().jb_solver_pass_name(self._handle, i).decode()
                 for i in range(npass.value)]
        return {n: ms[i] for i, n in enumerate(names)}, nsteps.value

    def step(self, eps, res_dev=None):
        """One asynchronous iteration on the current stream (after set_load)."""
        _lib.check(_lib.lib().jb_solver_step(
            self._handle, ctypes.c_void_p(eps.data_ptr()),
            ctypes.c_void_p(res_dev.data_ptr() if res_dev is not None else 0),
            ctypes.c_void_p(A.stream_handle())))


def basic_scheme(green_op, local_op, avg_eps, num_iter, tol=0.0, eps=None):
    """Run the basic scheme for one or several load cases (rows of avg_eps)."""
    E = np.atleast_2d(np.asarray(avg_eps, dtype=np.float64))
    return BasicScheme(green_op, local_op, E.shape[0]).run(E, num_iter, tol, eps)


@dataclass
class MixedResult(_Outcome):
    eps: torch.Tensor          # (nload,) + grid + (s,), FP64 on the device
    residuals: np.ndarray      # (outer steps, nload): FP64 residual at each outer step
    outer_iterations: int
    fp32_iterations: int
    mean_tau: np.ndarray       # (nload, s)
    status: np.ndarray = None  # (nload,) int32, see _Outcome

    def mean_stress(self, mat0, avg_eps):
        return _c0_apply(mat0, np.atleast_2d(avg_eps)) + self.mean_tau


class MixedScheme:
    """Mixed-precision basic scheme: FP32 bulk iterations with FP64 defect
    correction (no counterpart in the reference, whose loop is FP64).

    Every outer step evaluates the FP64 residual r = E - eps - Gamma0[(C -
    C0):eps] (whose normalised norm is the stopping test, as for
    BasicScheme), solves the correction equation d + Gamma0[(C - C0):d] = r
    approximately in FP32 and adds d to the FP64 strain field.  The inner
    solver is ``method="basic"`` (``inner - 1`` basic iterations from d = r)
    or ``method="bicgstab"`` (up to ``inner`` BiCGSTAB iterations from
    d = 0, sized after the first correction by the residual reduction rate
    seen over the previous one; ``"bicgstab_fixed"`` always runs ``inner``):
    the Krylov route of the reference's examples/square_inclusion_scipy.py,
    which hands the same operator to scipy's gmres.  The FP32 operators are
    built from the given FP64 ones (same material, grid, discretisation and
    phase map).  ``inner_dtype=torch.float64`` runs the same algorithm with
    FP64 corrections (the given operators serve both levels): the control
    that separates the gain of the inner solver from that of precision."""

    METHODS = {"basic": 0, "bicgstab": 1, "bicgstab_fixed": 2}

    def __init__(self, green_op, local_op, nload=1, inner=20, method="basic",
                 inner_dtype=torch.float32):
        if isinstance(local_op, _BlockDiagonalOperator):
            local = local_op.local
        else:
            local = local_op
        if not isinstance(local, LocalPhaseOperator):
            raise ValueError("the solver needs isotropic local operators (phase map)")
        if green_op.dtype != torch.float64 or local.dtype != torch.float64:
            raise ValueError("MixedScheme takes the FP64 operators")
        self.green_op = green_op
        self.local = local
        self.nload = int(nload)
        self.inner = int(inner)
        if inner_dtype == torch.float64:
            self.green32, self.local32 = green_op, local
        elif inner_dtype == torch.float32:
            self.green32 = type(green_op)(green_op.green, green_op.ishape[:-1], green_op.h,
                                          dtype=torch.float32)
            self.local32 = local.with_dtype(torch.float32)
        else:
            raise ValueError("inner_dtype must be torch.float32 or torch.float64")
        self.inner_dtype = inner_dtype
        if method not in self.METHODS:
            raise ValueError("method must be 'basic', 'bicgstab' or 'bicgstab_fixed'")
        self.method = method
        self._handle = ctypes.c_void_p()
        _lib.check(_lib.lib().jb_mixed_create(green_op.handle, local.handle, self.green32.handle,
                                              self.local32.handle, self.nload,
                                              ctypes.byref(self._handle)))
        _lib.check(_lib.lib().jb_mixed_set_method(self._handle, self.METHODS[method]))

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().jb_mixed_destroy(h)
            except Exception:
                pass
            self._handle = None

    @property
    def field_shape(self):
        return (self.nload,) + tuple(self.green_op.ishape)

    def run(self, avg_eps, tol, max_outer=1000, eps=None, inner=None):
        E = np.ascontiguousarray(np.asarray(avg_eps, dtype=np.float64).reshape(
            self.nload, self.green_op.ishape[-1]))
        init = eps is None
        if eps is None:
            eps = torch.empty(self.field_shape, dtype=torch.float64, device=A.device())
        elif tuple(eps.shape) != self.field_shape or eps.dtype != torch.float64 or \
                not eps.is_contiguous() or eps.device.type != "cuda":
            raise ValueError("eps must be a contiguous FP64 CUDA tensor of shape {0}".format(
                self.field_shape))
        inner = self.inner if inner is None else int(inner)
        res = np.zeros((max(int(max_outer), 1), self.nload))
        outer = ctypes.c_int(0)
        fp32 = ctypes.c_int(0)
        mean = np.zeros((self.nload, self.green_op.ishape[-1]))
        status = np.zeros(self.nload, dtype=np.int32)
        P = ctypes.POINTER(ctypes.c_double)
        _lib.check(_lib.lib().jb_mixed_run(self._handle, E.ctypes.data_as(P),
                                           ctypes.c_void_p(eps.data_ptr()),
                                           int(init), int(max_outer), inner, float(tol),
                                           res.ctypes.data_as(P), ctypes.byref(outer),
                                           ctypes.byref(fp32), mean.ctypes.data_as(P),
                                           status.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
                                           ctypes.c_void_p(A.stream_handle())))
        n = outer.value
        return MixedResult(eps=eps, residuals=res[:n].copy(), outer_iterations=n,
                           fp32_iterations=fp32.value, mean_tau=mean, status=status)


@dataclass
class GMRESResult(_Outcome):
    eps: torch.Tensor          # (nload,) + grid + (s,), FP64 on the device
    residuals: np.ndarray      # (iterations, nload): Givens estimate after each Arnoldi step
    final_residuals: np.ndarray  # (nload,): true residual at exit
    iterations: int            # Arnoldi steps (operator applications besides restarts)
    mean_tau: np.ndarray       # (nload, s)
    status: np.ndarray = None  # (nload,) int32, see _Outcome

    def mean_stress(self, mat0, avg_eps):
        return _c0_apply(mat0, np.atleast_2d(avg_eps)) + self.mean_tau


class GMRES:
    """Restarted GMRES(``restart``) on (I + Gamma0 (C - C0)) eps = E, FP64,
    with the Krylov basis on the device: the reference's Krylov route,
    examples/square_inclusion_scipy.py:52-59, 88, which hands this operator
    to scipy's gmres.  Every load case (rows of E) has its own Krylov space;
    the stopping test is the basic scheme's residual ||E - A eps|| /
    (sqrt(N) ||E||) <= tol, checked on the true residual at each restart.
    The basis holds restart + 1 fields of nload x grid x s doubles."""

    def __init__(self, green_op, local_op, nload=1, restart=20):
        if isinstance(local_op, _BlockDiagonalOperator):
            local = local_op.local
        else:
            local = local_op
        if not isinstance(local, LocalPhaseOperator):
            raise ValueError("the solver needs phase-map or field local operators")
        if green_op.dtype != torch.float64 or local.dtype != torch.float64:
            raise ValueError("GMRES takes FP64 operators")
        if tuple(local.shape) != tuple(green_op.ishape[:-1]):
            raise ValueError("local and green operators must share the grid")
        self.green_op = green_op
        self.local = local
        self.nload = int(nload)
        self.restart = int(restart)
        self._handle = ctypes.c_void_p()
        _lib.check(_lib.lib().jb_gmres_create(green_op.handle, local.handle, self.nload,
                                              self.restart, ctypes.byref(self._handle)))

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().jb_gmres_destroy(h)
            except Exception:
                pass
            self._handle = None

    @property
    def field_shape(self):
        return (self.nload,) + tuple(self.green_op.ishape)

    def run(self, avg_eps, tol=1e-8, max_iter=1000, eps=None, init=None):
        """eps (device FP64 tensor of field_shape) is the initial guess and is
        updated in place; if omitted, a new field set to E is used."""
        E = np.ascontiguousarray(np.asarray(avg_eps, dtype=np.float64).reshape(
            self.nload, self.green_op.ishape[-1]))
        if eps is None:
            eps = torch.empty(self.field_shape, dtype=torch.float64, device=A.device())
            init = True if init is None else init
        elif tuple(eps.shape) != self.field_shape or eps.dtype != torch.float64 or \
                not eps.is_contiguous() or eps.device.type != "cuda":
            raise ValueError("eps must be a contiguous FP64 CUDA tensor of shape {0}".format(
                self.field_shape))
        res = np.zeros((max(int(max_iter), 1), self.nload))
        final = np.zeros(self.nload)
        it = ctypes.c_int(0)
        mean = np.zeros((self.nload, self.green_op.ishape[-1]))
        status = np.zeros(self.nload, dtype=np.int32)
        P = ctypes.POINTER(ctypes.c_double)
        _lib.check(_lib.lib().jb_gmres_run(
            self._handle, E.ctypes.data_as(P), ctypes.c_void_p(eps.data_ptr()),
            int(bool(init)), int(max_iter), float(tol), res.ctypes.data_as(P),
            ctypes.byref(it), final.ctypes.data_as(P), mean.ctypes.data_as(P),
            status.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
            ctypes.c_void_p(A.stream_handle())))
        n = it.value
        return GMRESResult(eps=eps, residuals=res[:n].copy(), final_residuals=final,
                           iterations=n, mean_tau=mean, status=status)


class LippmannSchwingerOperator:
    """x -> x + Gamma0[(C - C0):x] on flattened host vectors (FP64), the
    matvec of the reference's examples/square_inclusion_scipy.py:52-59
    (``rmatvec``: x + (C - C0):Gamma0[x]), evaluated on the GPU; hand it to
    ``scipy.sparse.linalg.aslinearoperator`` and scipy's Krylov solvers."""

    def __init__(self, green_op, local_op):
        local = local_op.local if isinstance(local_op, _BlockDiagonalOperator) else local_op
        if not isinstance(local, LocalPhaseOperator):
            raise ValueError("the operator needs phase-map or field local operators")
        if green_op.dtype != torch.float64 or local.dtype != torch.float64:
            raise ValueError("LippmannSchwingerOperator takes FP64 operators")
        self.green_op = green_op
        self.local = local
        self.grid_shape = tuple(green_op.ishape)
        n = int(np.prod(self.grid_shape))
        self.shape = (n, n)
        self.dtype = np.dtype(np.float64)

    def _dev(self, x):
        return torch.from_numpy(np.ascontiguousarray(x, dtype=np.float64).reshape(
            self.grid_shape)).to(A.device())

    def matvec(self, x):
        xd = self._dev(x)
        t = torch.empty_like(xd)
        self.local.apply_device(xd, t)
        self.green_op._apply_device(t, t)
        return (xd + t).cpu().numpy().reshape(np.shape(x))

    def rmatvec(self, x):
        xd = self._dev(x)
        g = torch.empty_like(xd)
        self.green_op._apply_device(xd, g)
        t = torch.empty_like(xd)
        self.local.apply_device(g, t)
        return (xd + t).cpu().numpy().reshape(np.shape(x))
