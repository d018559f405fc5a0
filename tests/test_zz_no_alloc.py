"""rhmc_true_residuals_noalloc: the FP64 true-residual check for callers that must not allocate
device memory at that point (a program whose own pool owns all device memory, a chain sharing
the GPU under a fixed memory budget).  It must give the values of rhmc_true_residuals, which
takes its scratch from the context's workspace, call after call although its fixed scratch
array keeps the previous call's contents; it must leave the device's free memory unchanged;
and it must refuse sizes beyond its fixed limit.  Collected last on purpose: if it fails, a
run that stops at the first failure has already run every other test."""
import ctypes

import numpy as np
import pytest

import rhmc_b200 as rb
from rhmc_b200 import fields as F

pytestmark = pytest.mark.gpu

_D = ctypes.POINTER(ctypes.c_double)


def _noalloc(ctx, x, b, shifts, nrhs):
    sh = np.ascontiguousarray(shifts, np.float64)
    out = np.zeros((nrhs, len(sh)), np.float64)
    lib = rb.lib()
    lib.rhmc_true_residuals_noalloc.argtypes = [ctypes.c_void_p, ctypes.c_int, _D, ctypes.c_int, ctypes.c_void_p,
                                                ctypes.c_void_p, _D]
    rc = lib.rhmc_true_residuals_noalloc(ctx.h, len(sh), sh.ctypes.data_as(_D), nrhs, ctypes.c_void_p(x.data_ptr()),
                                         ctypes.c_void_p(b.data_ptr()), out.ctypes.data_as(_D))
    return rc, out


def test_noalloc_matches_workspace_version_on_consecutive_calls():
    import torch
    from gpu_util import new_ctx, to_internal
    dims = (8, 8, 8, 8)
    ctx = new_ctx(dims, mass=0.05)
    ctx.set_gauge(F.random_links(dims, seed=901))
    shifts = np.array([0.0, 0.01, 0.5, 3.0])
    nrhs = 2
    b = to_internal(ctx, rb.LINKS_F64_18, F.random_spinor(dims, seed=902, n=nrhs))
    xs = [to_internal(ctx, rb.LINKS_F64_18, F.random_spinor(dims, seed=s, n=nrhs * len(shifts))) for s in (903, 904)]
    torch.cuda.synchronize()
    for x in xs:  # two calls in a row, different inputs: nothing stale may leak through
        ref = ctx.true_residuals(x, b, shifts, nrhs)
        rc, out = _noalloc(ctx, x, b, shifts, nrhs)
        assert rc == 0, rb.lib().rhmc_last_error()
        np.testing.assert_allclose(out, ref, rtol=1e-12, atol=0)


def test_noalloc_leaves_free_device_memory_unchanged():
    """On a fresh context whose workspace has never been used by a true-residual check, repeated
    calls do not change the device's free memory, while the workspace version does grow it."""
    import torch
    from gpu_util import new_ctx, to_internal
    dims = (8, 8, 8, 16)
    ctx = new_ctx(dims, mass=0.05)
    ctx.set_gauge(F.random_links(dims, seed=911))
    shifts = np.array([0.0, 0.2])
    b = to_internal(ctx, rb.LINKS_F64_18, F.random_spinor(dims, seed=912))
    x = to_internal(ctx, rb.LINKS_F64_18, F.random_spinor(dims, seed=913, n=len(shifts)))
    torch.cuda.synchronize()
    # the first call may load the library's kernels onto the device (module loading is lazy)
    rc, first = _noalloc(ctx, x, b, shifts, 1)
    assert rc == 0, rb.lib().rhmc_last_error()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(3):
        rc, out = _noalloc(ctx, x, b, shifts, 1)
        assert rc == 0, rb.lib().rhmc_last_error()
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0
        np.testing.assert_array_equal(out, first)
    ref = ctx.true_residuals(x, b, shifts, 1)  # grow-on-demand workspace: allocates
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] < free0
    np.testing.assert_allclose(first, ref, rtol=1e-12, atol=0)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    import torch
    from gpu_util import new_ctx, to_internal
    dims = (18, 18, 18, 24)  # 69,984 sites per parity > 65,536
    ctx = new_ctx(dims, mass=0.05)
    b = to_internal(ctx, rb.LINKS_F64_18, F.random_spinor(dims, seed=905))
    x = to_internal(ctx, rb.LINKS_F64_18, F.random_spinor(dims, seed=906))
    torch.cuda.synchronize()
    rc, _ = _noalloc(ctx, x, b, [0.1], 1)
    assert rc == -1  # RHMC_ERR_ARG
    assert b"scratch limit" in rb.lib().rhmc_last_error()
