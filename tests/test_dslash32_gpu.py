"""The 32^4 Dslash of the benchmark (Haar links seed 1001, Gaussian spinor seed 2002) against the
reference's own Deo/Doe (lib/Action/fermionmatrix.cc:8-97), compiled unmodified at 32^4 into
oracle/_ref/libref_b32.so, and the neighbour/phase tables against the reference's init_geo
(lib/Main/Geometry/geometry.cc:26-161) and make_shift_table (lib/Tools/Packer/packer.cc:415-439)
at that volume.

Tolerances (relative L2 norm of the difference): FP64 links (18 and 12 reals) 1e-13, FP32
links (18 and 12 reals) 1e-6, half links and per-site-scaled half spinors 2e-3; tables bit-exact.
"""
import numpy as np
import pytest

import rhmc_b200 as rb
from rhmc_b200 import fields as F
from conftest import rel_err

pytestmark = pytest.mark.gpu

DIMS = (32, 32, 32, 32)
TOL = {rb.LINKS_F64_18: 1e-13, rb.LINKS_F64_12: 1e-13, rb.LINKS_F32_18: 1e-6, rb.LINKS_F32_12: 1e-6, rb.LINKS_F16_12: 2e-3}


@pytest.fixture(scope="module")
def lattice32():
    import oracle
    try:
        ref = oracle.RefLib("b32")
    except FileNotFoundError:
        pytest.skip("reference harness libref_b32 not built")
    assert ref.dims == DIMS
    from gpu_util import new_ctx
    u = F.random_links(DIMS, seed=1001)
    x = F.random_spinor(DIMS, seed=2002)
    ref.set_links(u)
    ctx = new_ctx(DIMS, mass=0.01, beta=5.8)
    ctx.set_gauge(u)
    out = {"ctx": ctx, "ref": ref, "x": x, "deo": ref.deo(x), "doe": ref.doe(x)}
    del u
    yield out
    ctx.close()


def test_tables_bit_exact_32(lattice32):
    t, e = lattice32["ctx"].geometry()
    t0, e0 = lattice32["ref"].tables()
    assert np.array_equal(t, t0)
    assert np.array_equal(e, e0)
    assert np.array_equal(t, lattice32["ref"].shift_table())


@pytest.mark.parametrize("fmt", [rb.LINKS_F64_18, rb.LINKS_F64_12, rb.LINKS_F32_18, rb.LINKS_F32_12, rb.LINKS_F16_12])
def test_dslash_32_vs_reference(lattice32, fmt):
    from gpu_util import to_internal, from_internal, internal_buffer
    ctx = lattice32["ctx"]
    xin = to_internal(ctx, fmt, lattice32["x"])
    for parity, key in ((0, "deo"), (1, "doe")):
        out = internal_buffer(ctx, fmt)
        ctx.dslash(fmt, parity, out, xin)
        err = rel_err(from_internal(ctx, fmt, out), lattice32[key])
        assert err < TOL[fmt], (rb.FMT_NAMES[fmt], key, err)


def test_dslash_32_host_entry_vs_reference(lattice32):
    """The reference-facing host-buffer call the benchmark's end-to-end number uses."""
    ctx = lattice32["ctx"]
    x = lattice32["x"]
    out = np.zeros_like(x)
    ctx.dslash_host(1, out, x)
    assert rel_err(out, lattice32["doe"]) < 1e-13
    ctx.dslash_host(0, out, x)
    assert rel_err(out, lattice32["deo"]) < 1e-13
