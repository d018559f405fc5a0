"""Helpers for the GPU tests: device buffers (torch) in the library's internal layout."""
import numpy as np

import rhmc_b200 as rb


def new_ctx(dims, mass=0.1, beta=5.5, bc=0):
    import torch
    ctx = rb.Context(dims, mass=mass, beta=beta, ferm_temp_bc=bc)
    ctx.set_stream(torch.cuda.current_stream().cuda_stream)
    return ctx


def internal_buffer(ctx, fmt, n=1):
    import torch
    dt = torch.float64 if fmt in (rb.LINKS_F64_18, rb.LINKS_F64_12) else torch.float32
    return torch.zeros(n * rb.spinor_floats(fmt, ctx.Vh), dtype=dt, device="cuda")


def to_internal(ctx, fmt, x):
    """x: numpy complex (Vh,3) or (n,Vh,3) -> device internal buffer."""
    import torch
    x = np.ascontiguousarray(x, np.complex128)
    n = 1 if x.ndim == 2 else x.shape[0]
    buf = internal_buffer(ctx, fmt, n)
    ctx.spinor_to_internal(fmt, buf, x, n)
    return buf


def from_internal(ctx, fmt, buf, n=1):
    out = np.zeros((n, ctx.Vh, 3) if n > 1 else (ctx.Vh, 3), np.complex128)
    import torch
    torch.cuda.synchronize()
    ctx.spinor_from_internal(fmt, out, buf, n)
    return out
