"""The allocation-free Green operator entry point (jb_green_apply_noalloc),
called through the C ABI, against the handle-based jb_green_apply.

It serves callers that cannot allocate device memory (a fixed memory pool,
no cudaMalloc outside set-up, plug-ins handed only their buffers): all its
scratch lives in a static device array.  This file is collected last, so a
failure here comes after every other test has run."""
import ctypes

import numpy as np
import pytest
import torch

import janus_b200.material.elastic.linear.isotropic as material
from janus_b200 import _lib
from janus_b200.green import filtered, truncated

P64 = ctypes.POINTER(ctypes.c_int64)


def _noalloc(x, shape, h, g, nu, variant, y):
    L = _lib.lib()
    fn = L.jb_green_apply_noalloc
    fn.argtypes = [ctypes.c_int, P64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                   ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    dims = (ctypes.c_int64 * len(shape))(*shape)
    st = torch.cuda.current_stream().cuda_stream
    return fn(len(shape), dims, h, g, nu, variant, ctypes.c_void_p(x.data_ptr()),
              ctypes.c_void_p(y.data_ptr()), ctypes.c_void_p(st))


def _reference_apply(x, shape, h, g, nu, variant):
    fac = truncated if variant == _lib.JB_TRUNCATED else filtered
    op = fac(material.create(g, nu, len(shape)).green_operator(), shape, h)
    return op.apply(x.clone())


@pytest.mark.gpu
def test_noalloc_matches_green_apply_on_consecutive_calls():
    rng = np.random.default_rng(123)
    cases = [((40, 50, 60), 1.0, 0.75, 0.3, _lib.JB_FILTERED),
             ((200, 300), 0.5, 2.0, 0.25, _lib.JB_TRUNCATED),
             ((40, 50, 60), 1.0, 0.75, 0.3, _lib.JB_TRUNCATED)]
    for shape, h, g, nu, variant in cases:
        s = 3 if len(shape) == 2 else 6
        x = torch.from_numpy(rng.normal(size=shape + (s,))).cuda()
        y = torch.empty_like(x)
        assert _noalloc(x, shape, h, g, nu, variant, y) == 0, _lib.lib().jb_last_error()
        torch.cuda.synchronize()
        ref = _reference_apply(x, shape, h, g, nu, variant)
        scale = ref.abs().max().item()
        np.testing.assert_allclose(y.cpu().numpy(), ref.cpu().numpy(), rtol=1e-13,
                                   atol=1e-13 * scale)
    # in place, and a rejected oversize grid leaves a clear message
    x = torch.from_numpy(rng.normal(size=(64, 64, 3))).cuda()
    ref = _reference_apply(x, (64, 64), 1.0, 1.0, 0.3, _lib.JB_FILTERED)
    assert _noalloc(x, (64, 64), 1.0, 1.0, 0.3, _lib.JB_FILTERED, x) == 0
    torch.cuda.synchronize()
    np.testing.assert_allclose(x.cpu().numpy(), ref.cpu().numpy(), rtol=1e-13,
                               atol=1e-13 * ref.abs().max().item())
    big = torch.empty(1, dtype=torch.float64, device="cuda")
    assert _noalloc(big, (128, 128, 128), 1.0, 1.0, 0.3, 0, big) == _lib.JB_EINVAL
    assert b"static scratch" in _lib.lib().jb_last_error()


@pytest.mark.gpu
def test_noalloc_warm_call_leaves_free_device_memory_unchanged():
    """The point of the entry point: a warm call allocates nothing, so the
    device's free memory is the same before and after it."""
    rng = np.random.default_rng(7)
    shape = (48, 40, 36)
    x = torch.from_numpy(rng.normal(size=shape + (6,))).cuda()
    y = torch.empty_like(x)
    assert _noalloc(x, shape, 1.0, 0.75, 0.3, _lib.JB_FILTERED, y) == 0   # warm
    torch.cuda.synchronize()
    first = y.clone()
    free0, _ = torch.cuda.mem_get_info()
    assert _noalloc(x, shape, 1.0, 0.75, 0.3, _lib.JB_FILTERED, y) == 0
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0
    assert torch.equal(y, first)


@pytest.mark.gpu
def test_noalloc_rejects_host_pointers():
    x = np.zeros((16, 16, 3))
    dims = (ctypes.c_int64 * 2)(16, 16)
    fn = _lib.lib().jb_green_apply_noalloc
    fn.argtypes = [ctypes.c_int, P64, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                   ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
    fn.restype = ctypes.c_int
    r = fn(2, dims, 1.0, 1.0, 0.3, 0, ctypes.c_void_p(x.ctypes.data),
           ctypes.c_void_p(x.ctypes.data), None)
    assert r == _lib.JB_EINVAL
    assert b"device" in _lib.lib().jb_last_error()
