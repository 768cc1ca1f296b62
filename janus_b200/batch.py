"""Batched mixed-precision solves of many independent cells (grids of
uneven sizes), one CUDA graph launch per outer step.

No counterpart in the reference, whose loop (square_basic.py:83-97) solves
one cell at a time in FP64.  Each problem is a ``MixedScheme`` (FP32 bulk
iterations, FP64 defect correction) over its own grid and load cases; the
native ``jb_batch`` runtime evaluates every problem's first FP64 residual,
then runs the whole iteration as ONE CUDA graph launch: a while node whose
body is a decision kernel (residuals recorded, outcomes updated, converged
or stopped problems retired, on the device) followed by one if node per
problem holding its FP32 correction sweeps and next FP64 residual, so the
problems run concurrently and the host reads nothing back until the end.
``persistent=False`` keeps the per-step form (one graph launch per outer
step, residuals read back each step, the graph captured again when a
problem leaves); results are bitwise the same.
"""
from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _arrays as A
from . import _lib
from .solvers import MixedResult, MixedScheme


class BatchedMixedScheme:
    """problems: sequence of (green_op, local_op, nload) triples (FP64
    operators of janus_b200.green / operators, any grid size each).

    With method "bicgstab" every captured correction runs the full ``inner``
    BiCGSTAB iterations (a lone MixedScheme sizes them adaptively); the
    results equal one-by-one solves with method "bicgstab_fixed" bitwise."""

    def __init__(self, problems, inner=20, branches=8, method="basic", persistent=True):
        if not problems:
            raise ValueError("a batch needs at least one problem")
        self.schemes = [MixedScheme(g, l, nload, inner, method=method)
                        for g, l, nload in problems]
        self.inner = int(inner)
        handles = (ctypes.c_void_p * len(self.schemes))(
            *[s._handle.value for s in self.schemes])
        self._handle = ctypes.c_void_p()
        _lib.check(_lib.lib().jb_batch_create(len(self.schemes), handles, int(branches),
                                              ctypes.byref(self._handle)))
        _lib.check(_lib.lib().jb_batch_set_persistent(self._handle, int(bool(persistent))))
        self.graph_launches = 0

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().jb_batch_destroy(h)
            except Exception:
                pass
            self._handle = None

    def __len__(self):
        return len(self.schemes)

    def new_fields(self):
        return [torch.empty(s.field_shape, dtype=torch.float64, device=A.device())
                for s in self.schemes]

    def run(self, avg_eps, tol, max_outer=1000, eps=None, inner=None):
        """avg_eps: one (nload, s) array per problem.  Returns one
        MixedResult per problem (FP64 strain fields on the device)."""
        if len(avg_eps) != len(self.schemes):
            raise ValueError("one macroscopic strain array per problem")
        Es = []
        for s, E in zip(self.schemes, avg_eps):
            Es.append(np.ascontiguousarray(np.asarray(E, dtype=np.float64).reshape(
                s.nload, s.green_op.ishape[-1])))
        init = eps is None
        if eps is None:
            eps = self.new_fields()
        for s, e in zip(self.schemes, eps):
            if tuple(e.shape) != s.field_shape or e.dtype != torch.float64 or \
                    not e.is_contiguous() or e.device.type != "cuda":
                raise ValueError("eps must be contiguous FP64 CUDA tensors of the problems' "
                                 "field shapes")
        inner = self.inner if inner is None else int(inner)
        max_outer = int(max_outer)
        P = len(self.schemes)
        E_all = np.ascontiguousarray(np.concatenate([E.ravel() for E in Es]))
        ptrs = (ctypes.c_void_p * P)(*[e.data_ptr() for e in eps])
        sizes = [s.nload for s in self.schemes]
        res = np.zeros(sum(max_outer * L for L in sizes))
        outer = (ctypes.c_int * P)()
        fp32 = (ctypes.c_int * P)()
        mean = np.zeros(E_all.shape[0])
        status = np.zeros(sum(sizes), dtype=np.int32)
        launches = ctypes.c_int(0)
        Pd = ctypes.POINTER(ctypes.c_double)
        _lib.check(_lib.lib().jb_batch_run(
            self._handle, E_all.ctypes.data_as(Pd), ptrs, int(init), max_outer, inner,
            float(tol), res.ctypes.data_as(Pd), outer, fp32, mean.ctypes.data_as(Pd),
            ctypes.byref(launches), status.ctypes.data_as(ctypes.POINTER(ctypes.c_int)),
            ctypes.c_void_p(A.stream_handle())))
        self.graph_launches = launches.value
        out = []
        r0 = m0 = s0 = 0
        for i, s in enumerate(self.schemes):
            L, C = s.nload, s.green_op.ishape[-1]
            hist = res[r0:r0 + max_outer * L].reshape(max_outer, L)[:outer[i]].copy()
            out.append(MixedResult(eps=eps[i], residuals=hist, outer_iterations=outer[i],
                                   fp32_iterations=fp32[i],
                                   mean_tau=mean[m0:m0 + L * C].reshape(L, C).copy(),
                                   status=status[s0:s0 + L].copy()))
            r0 += max_outer * L
            m0 += L * C
            s0 += L
        return out
