"""Operators: local tensors and block-diagonal (voxel-wise) operators.

Mirrors ``janus.operators`` (janus/operators.pyx:53-890) for the hot path:

* ``AbstractOperator`` / ``AbstractLinearOperator`` with ``init_sizes``,
  ``apply`` and ``to_memoryview`` (113-192);
* ``isotropic_4(sph, dev, dim)`` and ``FourthRankIsotropicTensor{2,3}D``
  (53-67, 257-408); ``LinearOperator(a)`` (195-254) and
  ``FourthRankCubicTensor2D(t1111, t1122, t1212, theta)`` (411-450);
* ``AbstractStructuredOperator{2,3}D`` with ``init_shapes`` and ``apply``
  (452-614);
* ``block_diagonal_operator(loc)`` / ``BlockDiagonalOperator{2,3}D(loc)``
  (70-87, 617-716), applied on the GPU;
* ``block_diagonal_linear_operator(a)`` / ``BlockDiagonalLinearOperator{2,3}D``
  with ``apply`` and ``apply_transpose`` (90-110, 719-890), on the GPU.

Field-wide operators run in the native library; a ``BlockDiagonalOperator``
built from isotropic tensors becomes a phase map (one index per voxel) plus
a table of (tr, dev) coefficients, one built from other square linear local
operators (cubic tensors, ``LinearOperator``) a phase map plus a table of
their matrices; both are applied with the reference's arithmetic (bitwise
identical results) and both drive the solvers.  Single-vector ``apply`` calls of the local
tensors run in the library's host code with the reference's operation order.

Difference from the reference: block-diagonal operators copy ``loc`` / ``a``
to the device when they are built (the reference keeps a shallow reference);
``refresh()`` re-reads them.
"""
from __future__ import annotations

import ctypes
import math

import numpy as np
import torch

from . import _arrays as A
from . import _lib

_P = ctypes.POINTER(ctypes.c_double)


# ---------------------------------------------------------------------------
# shape checks with the messages of janus/utils/checkarray.pyx:3-53
# ---------------------------------------------------------------------------

def _check_1d(a, n0):
    s = A.shape_of(a)
    if len(s) != 1 or s[0] != n0:
        raise ValueError('invalid shape: expected ({0},), actual ({1},)'.format(
            n0, s[0] if len(s) == 1 else s))


def _out_1d(out, n0):
    if out is None:
        return np.empty((n0,), dtype=np.float64)
    _check_1d(out, n0)
    return out


def _check_2d(a, n0, n1):
    s = A.shape_of(a)
    if len(s) != 2 or s != (n0, n1):
        raise ValueError('invalid shape: expected ({0}, {1}), actual {2}'.format(n0, n1, s))


def _out_2d(out, n0, n1):
    if out is None:
        return np.empty((n0, n1), dtype=np.float64)
    _check_2d(out, n0, n1)
    return out


def _check_nd(a, shape):
    s = A.shape_of(a)
    if s != tuple(shape):
        exp = ", ".join(str(v) for v in shape)
        act = ", ".join(str(v) for v in s)
        raise ValueError('invalid shape: expected ({0}), actual ({1})'.format(exp, act))


# ---------------------------------------------------------------------------
# single-vector operators
# ---------------------------------------------------------------------------

class AbstractOperator:
    """General operator mapping arrays of size isize to size osize
    (operators.pyx:113-164)."""

    def __init__(self):
        self._isize = 0
        self._osize = 0

    isize = property(lambda self: self._isize)
    osize = property(lambda self: self._osize)

    def init_sizes(self, isize, osize):
        if isize <= 0:
            raise ValueError('isize should be > 0 (was {})'.format(isize))
        if osize <= 0:
            raise ValueError('osize should be > 0 (was {})'.format(osize))
        self._isize = int(isize)
        self._osize = int(osize)

    def _apply_host(self, x, y):
        pass

    def apply(self, x, y=None):
        x = np.asarray(x, dtype=np.float64)
        _check_1d(x, self.isize)
        y = _out_1d(y, self.osize)
        self._apply_host(x, y)
        return y[...]


class AbstractLinearOperator(AbstractOperator):
    """Linear operator with a matrix (operators.pyx:167-192)."""

    def _to_matrix(self):
        raise NotImplementedError

    def to_memoryview(self, out=None):
        out = _out_2d(out, self.osize, self.isize)
        out[...] = self._to_matrix()
        return out[...]


class FourthRankIsotropicTensor(AbstractLinearOperator):
    """T = sph J + dev K (operators.pyx:257-303).  Use isotropic_4()."""

    def __init__(self, sph, dev, dim):
        super().__init__()
        dim = int(dim)
        sym = (dim * (dim + 1)) // 2
        self.init_sizes(sym, sym)
        self._dim = dim
        self._sph = float(sph)
        self._dev = float(dev)
        self._tr = (self._sph - self._dev) / float(dim)

    dim = property(lambda self: self._dim)
    sph = property(lambda self: self._sph)
    dev = property(lambda self: self._dev)
    tr = property(lambda self: self._tr)

    def __repr__(self):
        return ('FourthRankIsotropicTensor(sph={0}, dev={1}, dim={2})'
                .format(self.sph, self.dev, self.dim))

    def _apply_host(self, x, y):
        xc = np.ascontiguousarray(x, dtype=np.float64)
        res = np.empty(self.osize)
        _lib.check(_lib.lib().jb_isotropic_apply(self._dim, self._sph, self._dev,
                                                 xc.ctypes.data_as(_P), res.ctypes.data_as(_P)))
        y[...] = res


class FourthRankIsotropicTensor2D(FourthRankIsotropicTensor):
    """2D specialisation (operators.pyx:306-340); in place allowed."""

    def _to_matrix(self):
        a = (self.sph + self.dev) / 2.0
        b = 0.5 * (self.sph - self.dev)
        return np.array([[a, b, 0.0], [b, a, 0.0], [0.0, 0.0, self.dev]])


class FourthRankIsotropicTensor3D(FourthRankIsotropicTensor):
    """3D specialisation (operators.pyx:343-408); in place allowed."""

    def _to_matrix(self):
        a = (self.sph + 2.0 * self.dev) / 3.0
        b = (self.sph - self.dev) / 3.0
        m = np.zeros((6, 6))
        m[:3, :3] = b
        for i in range(3):
            m[i, i] = a
        for i in range(3, 6):
            m[i, i] = self.dev
        return m


class LinearOperator(AbstractLinearOperator):
    """Matrix-based linear operator (operators.pyx:195-254); keeps a shallow
    reference to ``a`` like the reference."""

    def __init__(self, a):
        super().__init__()
        a = np.asarray(a, dtype=np.float64)
        if a.ndim != 2:
            raise ValueError('a must be a 2D array')
        self.init_sizes(a.shape[1], a.shape[0])
        self.a = a

    def _apply_host(self, x, y):
        # y[i] = 0; y[i] += a[i, j] * x[j] in j order (operators.pyx:209-214)
        for i in range(self.osize):
            acc = 0.0
            for j in range(self.isize):
                acc += float(self.a[i, j]) * float(x[j])
            y[i] = acc

    def apply_transpose(self, x, y=None):
        """operators.pyx:225-244"""
        x = np.asarray(x, dtype=np.float64)
        _check_1d(x, self.osize)
        y = _out_1d(y, self.isize)
        for j in range(self.isize):
            acc = 0.0
            for i in range(self.osize):
                acc += float(self.a[i, j]) * float(x[i])
            y[j] = acc
        return y[...]

    def _to_matrix(self):
        return np.array(self.a, dtype=np.float64)


class FourthRankCubicTensor2D(AbstractLinearOperator):
    """Fourth-rank tensor with cubic symmetry in 2D (plane strain), rotated
    by theta (operators.pyx:411-450), Mandel form."""

    def __init__(self, t1111, t1122, t1212, theta):
        super().__init__()
        self.init_sizes(3, 3)
        self.dim = 2
        # operators.pyx:417-425, same operation order
        c = math.cos(4 * theta)
        s = math.sin(4 * theta)
        aux = t1111 - t1122 - 2 * t1212
        self.t11 = 0.25 * (3 * t1111 + t1122 + 2 * t1212 + c * aux)
        self.t12 = 0.25 * (t1111 + 3 * t1122 - 2 * t1212 - c * aux)
        self.t13 = 0.25 * math.sqrt(2.0) * s * aux
        self.t23 = -self.t13
        self.t33 = 0.50 * (t1111 - t1122 + 2 * t1212 - c * aux)

    def _apply_host(self, x, y):
        x0, x1, x2 = float(x[0]), float(x[1]), float(x[2])
        y[0] = self.t11 * x0 + self.t12 * x1 + self.t13 * x2
        y[1] = self.t12 * x0 + self.t11 * x1 + self.t23 * x2
        y[2] = self.t13 * x0 + self.t23 * x1 + self.t33 * x2

    def _to_matrix(self):
        return np.array([[self.t11, self.t12, self.t13],
                         [self.t12, self.t11, self.t23],
                         [self.t13, self.t23, self.t33]])


def isotropic_4(sph, dev, dim):
    """Create a FourthRankIsotropicTensor (operators.pyx:53-67)."""
    if dim == 2:
        return FourthRankIsotropicTensor2D(sph, dev, dim)
    elif dim == 3:
        return FourthRankIsotropicTensor3D(sph, dev, dim)
    raise ValueError('dim must be 2 or 3 (was {0})'.format(dim))


# ---------------------------------------------------------------------------
# structured (field) operators
# ---------------------------------------------------------------------------

class _AbstractStructuredOperator:
    _ndim = None

    def __init__(self):
        self._shape = None
        self._ishape = None
        self._oshape = None

    dim = property(lambda self: self._ndim)
    ishape = property(lambda self: self._ishape)
    oshape = property(lambda self: self._oshape)
    shape0 = property(lambda self: self._shape[0])
    shape1 = property(lambda self: self._shape[1])

    def _init(self, grid, ilast, olast):
        names = ["shape0", "shape1", "shape2"][:len(grid)]
        last = "ishape{}".format(len(grid)), "oshape{}".format(len(grid))
        for name, v in zip(names, grid):
            if v <= 0:
                raise ValueError('{} should be > 0 (was {})'.format(name, v))
        if ilast <= 0:
            raise ValueError('{} should be > 0 (was {})'.format(last[0], ilast))
        if olast <= 0:
            raise ValueError('{} should be > 0 (was {})'.format(last[1], olast))
        self._shape = tuple(int(v) for v in grid)
        self._ishape = self._shape + (int(ilast),)
        self._oshape = self._shape + (int(olast),)

    # device dtype of the operator (float64 unless built otherwise)
    _dtype = torch.float64

    def _apply_device(self, x, y):
        raise NotImplementedError

    def apply(self, x, y=None):
        """Return the image of x (stored in y if given), as the reference's
        AbstractStructuredOperator{2,3}D.apply (operators.pyx:509-528,
        592-614).  numpy in -> numpy out; CUDA tensors stay on the GPU."""
        _check_nd(x, self._ishape)
        if y is not None:
            _check_nd(y, self._oshape)
        xd = A.to_device(x, self._dtype)
        out = A.Output(y, self._oshape, self._dtype, x)
        self._apply_device(xd, out.target)
        if out.host:
            # the result goes back to the host (a synchronisation anyway):
            # a kernel that gave up a bounded wait invalidates it
            _lib.check_device(type(self).__name__ + ".apply")
        return out.finish()


class AbstractStructuredOperator2D(_AbstractStructuredOperator):
    """Operator on (shape0, shape1, ishape2) fields (operators.pyx:452-528)."""
    _ndim = 2
    ishape2 = property(lambda self: self._ishape[2])
    oshape2 = property(lambda self: self._oshape[2])

    def init_shapes(self, shape0, shape1, ishape2, oshape2):
        self._init((shape0, shape1), ishape2, oshape2)


class AbstractStructuredOperator3D(_AbstractStructuredOperator):
    """Operator on (shape0, shape1, shape2, ishape3) fields
    (operators.pyx:531-614)."""
    _ndim = 3
    shape2 = property(lambda self: self._shape[2])
    ishape3 = property(lambda self: self._ishape[3])
    oshape3 = property(lambda self: self._oshape[3])

    def init_shapes(self, shape0, shape1, shape2, ishape3, oshape3):
        self._init((shape0, shape1, shape2), ishape3, oshape3)


class LocalPhaseOperator:
    """Device form of (C - C0):eps on a phase map: the native handle plus
    the phase map, for the solver and the block-diagonal operators.

    ``phase=None`` makes it a stiffness field: ``sph`` and ``dev`` then hold
    one coefficient per voxel (C order over the grid), as for mu(x).
    ``matrices`` (nphase x s x s) replaces (sph, dev) by a full matrix per
    entry (anisotropic phases, e.g. rotated cubic grains)."""

    def __init__(self, dim, shape, phase, sph, dev, dtype=torch.float64, matrices=None):
        self.dim = int(dim)
        self.shape = tuple(int(v) for v in shape)
        self.dtype = dtype
        self.matrices = None
        if matrices is not None:
            self._init_matrices(phase, matrices)
            return
        if A.is_tensor(sph):
            sph = sph.detach().cpu().numpy()
        if A.is_tensor(dev):
            dev = dev.detach().cpu().numpy()
        sph = np.ascontiguousarray(np.asarray(sph, dtype=np.float64).ravel())
        dev = np.ascontiguousarray(np.asarray(dev, dtype=np.float64).ravel())
        if sph.shape != dev.shape:
            raise ValueError("sph and dev must have the same length")
        self.nphase = int(sph.shape[0])
        self.sph = sph
        self.dev = dev
        if phase is None:
            nvox = int(np.prod(self.shape))
            if self.nphase != nvox:
                raise ValueError("a stiffness field needs one (sph, dev) pair per voxel "
                                 "({} given for {} voxels)".format(self.nphase, nvox))
            self.phase = None
            self._handle = ctypes.c_void_p()
            _lib.check(_lib.lib().jb_local_create(
                self.dim, _lib.i64_array(self.shape), self.nphase, sph.ctypes.data_as(_P),
                dev.ctypes.data_as(_P), None, 0, A.jb_dtype(dtype),
                ctypes.byref(self._handle)))
            return
        index_bytes = 1 if self.nphase <= 256 else 4
        if A.is_tensor(phase):
            ph = phase.to(A.device())
        else:
            ph = torch.from_numpy(np.ascontiguousarray(np.asarray(phase))).to(A.device())
        if tuple(ph.shape) != self.shape:
            raise ValueError("phase map shape {} differs from grid {}".format(
                tuple(ph.shape), self.shape))
        if ph.numel() and (int(ph.min()) < 0 or int(ph.max()) >= self.nphase):
            raise ValueError("phase indices must lie in [0, {})".format(self.nphase))
        ph = ph.to(torch.uint8 if index_bytes == 1 else torch.int32).contiguous()
        self.phase = ph
        self._handle = ctypes.c_void_p()
        _lib.check(_lib.lib().jb_local_create(
            self.dim, _lib.i64_array(self.shape), self.nphase, sph.ctypes.data_as(_P),
            dev.ctypes.data_as(_P), ctypes.c_void_p(ph.data_ptr()), index_bytes,
            A.jb_dtype(dtype), ctypes.byref(self._handle)))

    def _init_matrices(self, phase, matrices):
        s = 3 if self.dim == 2 else 6
        mats = np.ascontiguousarray(np.asarray(matrices, dtype=np.float64))
        if mats.ndim != 3 or mats.shape[1:] != (s, s):
            raise ValueError("matrices must have shape (nphase, {0}, {0})".format(s))
        self.matrices = mats
        self.sph = self.dev = None
        self.nphase = int(mats.shape[0])
        P = ctypes.POINTER(ctypes.c_double)
        self._handle = ctypes.c_void_p()
        if phase is None:
            if self.nphase != int(np.prod(self.shape)):
                raise ValueError("a matrix field needs one matrix per voxel")
            self.phase = None
            _lib.check(_lib.lib().jb_local_create_matrix(
                self.dim, _lib.i64_array(self.shape), self.nphase, mats.ctypes.data_as(P), None,
                0, A.jb_dtype(self.dtype), ctypes.byref(self._handle)))
            return
        index_bytes = 1 if self.nphase <= 256 else 4
        ph = self._phase_map(phase, index_bytes)
        _lib.check(_lib.lib().jb_local_create_matrix(
            self.dim, _lib.i64_array(self.shape), self.nphase, mats.ctypes.data_as(P),
            ctypes.c_void_p(ph.data_ptr()), index_bytes, A.jb_dtype(self.dtype),
            ctypes.byref(self._handle)))

    def _phase_map(self, phase, index_bytes):
        if A.is_tensor(phase):
            ph = phase.to(A.device())
        else:
            ph = torch.from_numpy(np.ascontiguousarray(np.asarray(phase))).to(A.device())
        if tuple(ph.shape) != self.shape:
            raise ValueError("phase map shape {} differs from grid {}".format(
                tuple(ph.shape), self.shape))
        if ph.numel() and (int(ph.min()) < 0 or int(ph.max()) >= self.nphase):
            raise ValueError("phase indices must lie in [0, {})".format(self.nphase))
        ph = ph.to(torch.uint8 if index_bytes == 1 else torch.int32).contiguous()
        self.phase = ph
        return ph

    def with_dtype(self, dtype):
        """The same operator in another precision."""
        if self.matrices is not None:
            return LocalPhaseOperator(self.dim, self.shape, self.phase, None, None, dtype,
                                      matrices=self.matrices)
        return LocalPhaseOperator(self.dim, self.shape, self.phase, self.sph, self.dev, dtype)

    @property
    def handle(self):
        return self._handle

    def apply_device(self, x, y, batch=1):
        _lib.check(_lib.lib().jb_local_apply(self._handle, ctypes.c_void_p(x.data_ptr()),
                                             ctypes.c_void_p(y.data_ptr()), int(batch),
                                             ctypes.c_void_p(A.stream_handle())))

    def __del__(self):
        h = getattr(self, "_handle", None)
        if h is not None and h.value:
            try:
                _lib.lib().jb_local_destroy(h)
            except Exception:
                pass
            self._handle = None


def _block_linear(a_dev, x, y, osz, isz, transpose, dtype):
    nvox = a_dev.shape[0]
    _lib.check(_lib.lib().jb_block_linear_apply(
        A.jb_dtype(dtype), int(nvox), int(osz), int(isz), ctypes.c_void_p(a_dev.data_ptr()),
        ctypes.c_void_p(x.data_ptr()), ctypes.c_void_p(y.data_ptr()), int(transpose),
        ctypes.c_void_p(A.stream_handle())))


class _BlockDiagonalOperator:
    """Shared implementation of BlockDiagonalOperator2D/3D."""

    def _build(self, loc, dtype):
        if loc is None:
            raise ValueError('loc should not be None')
        loc = np.asarray(loc, dtype=object)
        if loc.ndim != self._ndim:
            raise ValueError('loc must be a {0}D array of operators'.format(self._ndim))
        first = loc[(0,) * self._ndim]
        self.init_shapes(*loc.shape, first.isize, first.osize)
        self._dtype = A.torch_dtype(dtype)
        self.loc = loc
        self.refresh()

    def refresh(self):
        """(Re)build the device form of the local operators from ``loc``
        with the checks of operators.pyx:639-653 / 689-704."""
        loc = self.loc
        ilast, olast = self._ishape[-1], self._oshape[-1]
        flat = loc.ravel()
        keys = {}
        ops = []
        phase = np.empty(flat.shape[0], dtype=np.int64)
        iso = True
        for v, op in enumerate(flat):
            if op.isize != ilast:
                raise ValueError('invalid dimension block operator input: expected {0}, '
                                 'actual {1}'.format(ilast, op.isize))
            if op.osize != olast:
                raise ValueError('invalid dimension block operator output: expected {0}, '
                                 'actual {1}'.format(olast, op.osize))
            if isinstance(op, FourthRankIsotropicTensor) and op.dim == self._ndim:
                key = ("iso", op.sph, op.dev)
            else:
                iso = False
                key = ("obj", id(op))
            p = keys.get(key)
            if p is None:
                p = len(ops)
                keys[key] = p
                ops.append(op)
            phase[v] = p
        phase = phase.reshape(loc.shape)
        self._local = None
        self._matrices = None
        if iso:
            self._local = LocalPhaseOperator(self._ndim, self._shape, phase,
                                             [op.sph for op in ops], [op.dev for op in ops],
                                             self._dtype)
        else:
            mats = []
            for op in ops:
                if not hasattr(op, "to_memoryview"):
                    raise TypeError("local operators must be linear (define to_memoryview)")
                mats.append(np.asarray(op.to_memoryview(), dtype=np.float64))
            if ilast == olast and ilast == (3 if self._ndim == 2 else 6):
                # square Mandel blocks: a phase map + matrix table (solver-ready)
                self._local = LocalPhaseOperator(self._ndim, self._shape, phase, None, None,
                                                 self._dtype, matrices=np.stack(mats))
            else:
                table = torch.from_numpy(np.stack(mats)).to(A.device(), self._dtype)
                idx = torch.from_numpy(phase.ravel()).to(A.device())
                self._matrices = table[idx].contiguous()

    @classmethod
    def from_phases(cls, phase, ops, dtype=None):
        """Build from a phase map (integer array of the grid shape) and the
        list of isotropic local tensors it indexes: the fast constructor for
        large grids (no per-voxel Python objects)."""
        obj = cls.__new__(cls)
        _AbstractStructuredOperator.__init__(obj)
        phase_shape = A.shape_of(phase)
        if len(phase_shape) != cls._ndim:
            raise ValueError('phase map must be {0}D'.format(cls._ndim))
        op0 = ops[0]
        obj.init_shapes(*phase_shape, op0.isize, op0.osize)
        obj._dtype = A.torch_dtype(dtype)
        obj.loc = None
        obj._matrices = None
        if all(isinstance(op, FourthRankIsotropicTensor) and op.dim == cls._ndim
               for op in ops):
            obj._local = LocalPhaseOperator(cls._ndim, phase_shape, phase,
                                            [op.sph for op in ops], [op.dev for op in ops],
                                            obj._dtype)
            return obj
        s = 3 if cls._ndim == 2 else 6
        mats = []
        for op in ops:
            if not hasattr(op, "to_memoryview") or op.isize != s or op.osize != s:
                raise TypeError("from_phases expects {0} x {0} linear local operators".format(s))
            mats.append(np.asarray(op.to_memoryview(), dtype=np.float64))
        obj._local = LocalPhaseOperator(cls._ndim, phase_shape, phase, None, None, obj._dtype,
                                        matrices=np.stack(mats))
        return obj

    @property
    def local(self):
        """The phase-map device operator (None for general local operators)."""
        return self._local

    def _apply_device(self, x, y):
        if self._local is not None:
            self._local.apply_device(x, y)
        else:
            s = self._ishape[-1]
            _block_linear(self._matrices, x, y, self._oshape[-1], s, 0, self._dtype)


class BlockDiagonalOperator2D(_BlockDiagonalOperator, AbstractStructuredOperator2D):
    """Block-diagonal operator on 2D grids (operators.pyx:617-664)."""

    def __init__(self, loc, dtype=None):
        AbstractStructuredOperator2D.__init__(self)
        self._build(loc, dtype)


class BlockDiagonalOperator3D(_BlockDiagonalOperator, AbstractStructuredOperator3D):
    """Block-diagonal operator on 3D grids (operators.pyx:667-716)."""

    def __init__(self, loc, dtype=None):
        AbstractStructuredOperator3D.__init__(self)
        self._build(loc, dtype)


def block_diagonal_operator(loc):
    """Create a block-diagonal operator from a 2D/3D array of local
    operators (operators.pyx:70-87)."""
    dim = len(np.asarray(loc, dtype=object).shape)
    if dim == 2:
        return BlockDiagonalOperator2D(loc)
    elif dim == 3:
        return BlockDiagonalOperator3D(loc)
    raise ValueError('number of dimensions of loc must be 2 or 3 (was {0})'.format(dim))


class _BlockDiagonalLinearOperator:
    def _build(self, a, dtype):
        if a is None:
            raise ValueError('a should not be None')
        s = A.shape_of(a)
        if len(s) != self._ndim + 2:
            raise ValueError('a must have {0} dimensions'.format(self._ndim + 2))
        if s[-1] > 8 or s[-2] > 8:
            raise ValueError('local blocks larger than 8 x 8 are not supported')
        # operators.pyx:734, 817: ishape = a.shape[-1], oshape = a.shape[-2]
        self.init_shapes(*s[:-2], s[-1], s[-2])
        self._dtype = A.torch_dtype(dtype)
        self.a = a
        self.refresh()

    def refresh(self):
        self._a = A.to_device(self.a, self._dtype).reshape(
            -1, self._oshape[-1], self._ishape[-1])

    def _apply_device(self, x, y):
        _block_linear(self._a, x, y, self._oshape[-1], self._ishape[-1], 0, self._dtype)

    def apply_transpose(self, x, y=None):
        """y[v] = a[v]^T x[v] (operators.pyx:776-799, 863-890)."""
        _check_nd(x, self._oshape)
        if y is not None:
            _check_nd(y, self._ishape)
        xd = A.to_device(x, self._dtype)
        out = A.Output(y, self._ishape, self._dtype, x)
        _block_linear(self._a, xd, out.target, self._oshape[-1], self._ishape[-1], 1,
                      self._dtype)
        return out.finish()


class BlockDiagonalLinearOperator2D(_BlockDiagonalLinearOperator, AbstractStructuredOperator2D):
    """Per-voxel matrices on a 2D grid (operators.pyx:719-799)."""

    def __init__(self, a, dtype=None):
        AbstractStructuredOperator2D.__init__(self)
        self._build(a, dtype)


class BlockDiagonalLinearOperator3D(_BlockDiagonalLinearOperator, AbstractStructuredOperator3D):
    """Per-voxel matrices on a 3D grid (operators.pyx:802-890)."""

    def __init__(self, a, dtype=None):
        AbstractStructuredOperator3D.__init__(self)
        self._build(a, dtype)


def block_diagonal_linear_operator(a):
    """Create a block-diagonal linear operator from a 4D/5D array of local
    matrices (operators.pyx:90-110)."""
    dim = len(A.shape_of(a)) - 2
    if dim == 2:
        return BlockDiagonalLinearOperator2D(a)
    elif dim == 3:
        return BlockDiagonalLinearOperator3D(a)
    raise ValueError('number of dimensions of a must be 4 or 5 (was {0})'.format(dim))
