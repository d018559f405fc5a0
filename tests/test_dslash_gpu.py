"""Geometry and Dslash on the B200 against the oracle (C restatement of
lib/Action/fermionmatrix.cc:8-97 and lib/Main/Geometry/geometry.cc:26-161).

Tolerances (relative L2 norm of the difference): FP64 links 1e-13, FP32 links 1e-6, half
precision links and spinors with per-site scales 2e-3 (11-bit significands).
"""
import numpy as np
import pytest

import rhmc_b200 as rb
from rhmc_b200 import fields as F
from conftest import rel_err

pytestmark = pytest.mark.gpu

DIMS = [(4, 4, 4, 4), (6, 4, 4, 8), (8, 8, 8, 8), (4, 6, 2, 10)]
TOL = {rb.LINKS_F64_18: 1e-13, rb.LINKS_F64_12: 1e-13, rb.LINKS_F32_18: 1e-6, rb.LINKS_F32_12: 1e-6, rb.LINKS_F16_12: 2e-3}


@pytest.fixture(scope="module")
def oracle_mod():
    import oracle
    return oracle


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("bc", [0, 1])
def test_geometry_bit_exact(dims, bc, oracle_mod):
    from gpu_util import new_ctx
    ctx = new_ctx(dims, bc=bc)
    t, e = ctx.geometry()
    orc = oracle_mod.Oracle(dims, bc)
    t0, e0 = orc.tables()
    assert np.array_equal(t, t0)
    assert np.array_equal(e, e0)


@pytest.mark.parametrize("dims", DIMS)
@pytest.mark.parametrize("fmt", [rb.LINKS_F64_18, rb.LINKS_F64_12, rb.LINKS_F32_18, rb.LINKS_F32_12, rb.LINKS_F16_12])
def test_dslash_vs_oracle(dims, fmt, oracle_mod):
    from gpu_util import new_ctx, to_internal, from_internal, internal_buffer
    ctx = new_ctx(dims)
    u = F.random_links(dims, seed=1001)
    ctx.set_gauge(u)
    orc = oracle_mod.Oracle(dims)
    x = F.random_spinor(dims, seed=2002)
    for parity in (0, 1):
        ref = orc.deo(u, x) if parity == 0 else orc.doe(u, x)
        xin = to_internal(ctx, fmt, x)
        out = internal_buffer(ctx, fmt)
        ctx.dslash(fmt, parity, out, xin)
        got = from_internal(ctx, fmt, out)
        assert rel_err(got, ref) < TOL[fmt], (parity, rel_err(got, ref))


@pytest.mark.parametrize("fmt", [rb.LINKS_F64_18, rb.LINKS_F32_12, rb.LINKS_F16_12])
@pytest.mark.parametrize("n", [2, 3, 4, 5, 8])
def test_dslash_multi_rhs_matches_single(fmt, n):
    from gpu_util import new_ctx, to_internal, from_internal, internal_buffer
    dims = (6, 4, 4, 8)
    ctx = new_ctx(dims)
    u = F.random_links(dims, seed=7)
    ctx.set_gauge(u)
    xs = F.random_spinor(dims, seed=8, n=n)
    xin = to_internal(ctx, fmt, xs)
    out = internal_buffer(ctx, fmt, n)
    ctx.dslash(fmt, 1, out, xin, n)
    got = from_internal(ctx, fmt, out, n)
    for r in range(n):
        xi = to_internal(ctx, fmt, xs[r])
        o1 = internal_buffer(ctx, fmt)
        ctx.dslash(fmt, 1, o1, xi)
        one = from_internal(ctx, fmt, o1)
        assert np.array_equal(one, got[r])


def test_mdagm_vs_oracle(oracle_mod):
    from gpu_util import new_ctx, to_internal, from_internal, internal_buffer
    dims = (6, 4, 4, 8)
    mass = 0.05
    ctx = new_ctx(dims, mass=mass)
    u = F.random_links(dims, seed=11)
    ctx.set_gauge(u)
    orc = oracle_mod.Oracle(dims)
    x = F.random_spinor(dims, seed=12)
    for shift in (0.0, 0.37):
        ref = orc.mdagm(u, x, mass, shift)
        xin = to_internal(ctx, rb.LINKS_F64_18, x)
        out = internal_buffer(ctx, rb.LINKS_F64_18)
        ctx.mdagm(rb.LINKS_F64_18, out, xin, shift)
        got = from_internal(ctx, rb.LINKS_F64_18, out)
        assert rel_err(got, ref) < 1e-13


@pytest.mark.parametrize("dims", [(4, 4, 4, 4), (4, 6, 2, 10), (4, 4, 2, 14), (4, 4, 4, 2), (2, 4, 2, 34), (8, 8, 8, 16)])
def test_dslash_host_reference_facing(oracle_mod, dims):
    """Host arrays in the reference's layout: uploaded, applied and downloaded in chunks of whole
    t-slabs, the largest count in [3, 16] that divides nt (4, 10, 14 and 16 chunks here); nt = 2
    and nt = 34 have no such count and run unchunked."""
    from gpu_util import new_ctx
    ctx = new_ctx(dims)
    u = F.random_links(dims, seed=21)
    ctx.set_gauge(u)
    orc = oracle_mod.Oracle(dims)
    x = F.random_spinor(dims, seed=22)
    out = np.zeros_like(x)
    ctx.dslash_host(1, out, x)
    assert rel_err(out, orc.doe(u, x)) < 1e-13
    ctx.dslash_host(0, out, x)
    assert rel_err(out, orc.deo(u, x)) < 1e-13
    # page-locked buffers: the output is stored into host memory by the kernels themselves
    import torch
    pin_in = torch.from_numpy(np.ascontiguousarray(x).view(np.float64).reshape(-1).copy()).pin_memory()
    pin_out = torch.zeros(pin_in.numel(), dtype=torch.float64).pin_memory()
    ctx.dslash_host(1, pin_out.numpy(), pin_in.numpy())
    got = pin_out.numpy().view(np.complex128).reshape(x.shape)
    assert rel_err(got, orc.doe(u, x)) < 1e-13
    ctx.dslash_host(0, pin_out.numpy(), pin_in.numpy())
    got = pin_out.numpy().view(np.complex128).reshape(x.shape)
    assert rel_err(got, orc.deo(u, x)) < 1e-13


def test_gauge_roundtrip_exact():
    from gpu_util import new_ctx
    dims = (4, 6, 2, 10)
    ctx = new_ctx(dims)
    u = F.random_links(dims, seed=31)
    ctx.set_gauge(u)
    assert np.array_equal(ctx.get_gauge(), u)


def test_antihermiticity_identity():
    """<y, Deo x> = -<Doe y, x> (D_eo = -D_oe^dag), an oracle-free check at a larger size."""
    from gpu_util import new_ctx, to_internal, from_internal, internal_buffer
    dims = (8, 8, 8, 16)
    ctx = new_ctx(dims)
    u = F.random_links(dims, seed=41)
    ctx.set_gauge(u)
    xo = F.random_spinor(dims, seed=42)
    ye = F.random_spinor(dims, seed=43)
    fmt = rb.LINKS_F64_18
    a = internal_buffer(ctx, fmt)
    ctx.dslash(fmt, 0, a, to_internal(ctx, fmt, xo))
    b = internal_buffer(ctx, fmt)
    ctx.dslash(fmt, 1, b, to_internal(ctx, fmt, ye))
    lhs = np.vdot(ye, from_internal(ctx, fmt, a))
    rhs = -np.vdot(from_internal(ctx, fmt, b), xo)
    assert abs(lhs - rhs) < 1e-10 * abs(lhs)


def test_half_spinor_roundtrip():
    """Half precision with a per-site scale keeps every site to 2^-11 of its largest component."""
    from gpu_util import new_ctx, to_internal, from_internal
    dims = (6, 4, 4, 8)
    ctx = new_ctx(dims)
    x = F.random_spinor(dims, seed=9) * np.geomspace(1e-6, 1e3, ctx.Vh)[:, None]  # per-site scales over 9 decades
    back = from_internal(ctx, rb.LINKS_F16_12, to_internal(ctx, rb.LINKS_F16_12, x))
    site_max = np.maximum(np.abs(x.real), np.abs(x.imag)).max(1)
    err = np.maximum(np.abs((back - x).real), np.abs((back - x).imag)).max(1)
    assert np.all(err <= site_max * 2.0 ** -11 * 1.01)


def test_half_spinor_tiny_sites_flush_to_zero():
    """Sites whose largest component is below the smallest normal float (1/scale would overflow)
    are stored as zero instead of inf/NaN; the Dslash of such a field stays finite."""
    from gpu_util import new_ctx, to_internal, from_internal, internal_buffer
    dims = (6, 4, 4, 8)
    ctx = new_ctx(dims)
    ctx.set_gauge(F.random_links(dims, seed=10))
    x = F.random_spinor(dims, seed=11)
    tiny = np.arange(ctx.Vh) % 3 == 0
    x[tiny] *= 1e-40
    xin = to_internal(ctx, rb.LINKS_F16_12, x)
    back = from_internal(ctx, rb.LINKS_F16_12, xin)
    assert np.all(np.isfinite(back))
    assert not np.any(back[tiny])
    normal = ~tiny
    assert rel_err(back[normal], x[normal]) < 2e-3
    out = internal_buffer(ctx, rb.LINKS_F16_12)
    ctx.dslash(rb.LINKS_F16_12, 1, out, xin)
    assert np.all(np.isfinite(from_internal(ctx, rb.LINKS_F16_12, out)))
