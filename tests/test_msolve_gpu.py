"""Multi-shift CG on the B200 against the oracle (restatement of multips_shifted_invert,
lib/Action/Inverter/inverter.cc:142-339) and against the reference's own CPU code.

Tolerances: FP64 mode reproduces the reference iteration (same recurrences, FP64, FMA
rounding only), so solutions agree to 1e-10 relative at residual 1e-10; mixed mode is checked
by the FP64 true residual of every system, which must be <= the requested residual (up to the
rounding of its evaluation, 1e-3 of it at 1e-10).
"""
import numpy as np
import pytest

import rhmc_b200 as rb
from rhmc_b200 import fields as F
from conftest import rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def oracle_mod():
    import oracle
    return oracle


def shifts_log(n, lo, hi):
    return np.geomspace(lo, hi, n)


@pytest.mark.parametrize("dims,mass", [((4, 4, 4, 4), 0.1), ((6, 4, 4, 8), 0.05)])
def test_msolve_fp64_vs_oracle(dims, mass, oracle_mod):
    from gpu_util import new_ctx
    ctx = new_ctx(dims, mass=mass)
    u = F.random_links(dims, seed=101)
    ctx.set_gauge(u)
    b = F.random_spinor(dims, seed=102)
    shifts = shifts_log(6, 1e-3, 10.0)
    x, info = ctx.msolve_host(b, shifts, 1e-10)
    orc = oracle_mod.Oracle(dims)
    xr, it = orc.msolve(u, b, mass, shifts, 1e-10)
    assert info["status"] == 0
    assert info["iters"][0] <= it
    for i in range(len(shifts)):
        assert rel_err(x[i], xr[i]) < 1e-10, (i, rel_err(x[i], xr[i]))


def test_msolve_fp64_vs_reference_code(oracle_mod):
    """The reference's own multips_shifted_invert (compiled CPU sources, 4^4, mass 0.1)."""
    try:
        ref = oracle_mod.RefLib("t4")
    except FileNotFoundError:
        pytest.skip("reference harness not built")
    from gpu_util import new_ctx
    dims = ref.dims
    ctx = new_ctx(dims, mass=ref.mass)
    u = F.random_links(dims, seed=111)
    ref.set_links(u)
    ctx.set_gauge(u)
    b = F.random_spinor(dims, seed=112, n=ref.no_ps)
    ref.set_chi(b)
    shifts = shifts_log(5, 2e-3, 30.0)
    xr = ref.msolve(1e-10, shifts)[0]
    x, info = ctx.msolve_host(b[0], shifts, 1e-10)
    for i in range(len(shifts)):
        assert rel_err(x[i], xr[i]) < 1e-10


def test_msolve_batched_rhs_identical():
    from gpu_util import new_ctx
    dims = (6, 4, 4, 8)
    ctx = new_ctx(dims, mass=0.05)
    ctx.set_gauge(F.random_links(dims, seed=121))
    bs = F.random_spinor(dims, seed=122, n=3)
    shifts = shifts_log(4, 1e-3, 1.0)
    xb, info = ctx.msolve_host(bs, shifts, 1e-10)
    for r in range(3):
        x1, _ = ctx.msolve_host(bs[r], shifts, 1e-10)
        assert np.array_equal(x1, xb[r])


@pytest.mark.parametrize("nrhs", [2, 4])
def test_msolve_fp32_packed_batch_identical(nrhs):
    """FP32 mode keeps a batch's base vectors packed (2 or 4 right-hand sides per element) and a
    single right-hand side's in plane layout: the two layouts run the same arithmetic per RHS,
    so each batched solution equals its single solve bit for bit."""
    from gpu_util import new_ctx
    dims = (6, 4, 4, 8)
    ctx = new_ctx(dims, mass=0.05)
    ctx.set_gauge(F.random_links(dims, seed=125))
    bs = F.random_spinor(dims, seed=126, n=nrhs)
    shifts = shifts_log(5, 1e-3, 2.0)
    xb, info = ctx.msolve_host(bs, shifts, 1e-5, mode=rb.MSOLVE_FP32, fmt=rb.LINKS_F32_12)
    assert info["status"] == 0, info
    for r in range(nrhs):
        x1, _ = ctx.msolve_host(bs[r], shifts, 1e-5, mode=rb.MSOLVE_FP32, fmt=rb.LINKS_F32_12)
        assert np.array_equal(x1, xb[r]), r


@pytest.mark.parametrize("fmt", [rb.LINKS_F32_12, rb.LINKS_F32_18, rb.LINKS_F16_12])
@pytest.mark.parametrize("nrhs", [1, 4, 5])
def test_msolve_mixed_true_residual(fmt, nrhs, oracle_mod):
    from gpu_util import new_ctx
    import torch
    dims = (8, 8, 8, 8)
    mass = 0.02
    ctx = new_ctx(dims, mass=mass)
    u = F.random_links(dims, seed=131)
    ctx.set_gauge(u)
    bs = F.random_spinor(dims, seed=132, n=nrhs)
    shifts = shifts_log(8, 1e-4, 50.0)
    res = 1e-10
    xm, info = ctx.msolve_host(bs if nrhs > 1 else bs[0], shifts, res, mode=rb.MSOLVE_MIXED, fmt=fmt)
    assert info["status"] == 0, info
    # the precision schedule handed over to FP32 with reliable updates, and left at most a few
    # systems for the refinement
    assert 0 < info["iters_fp64"] < info["iters_total"], info
    assert info["ms_reliable_updates"] > 0, info
    assert info["systems_refined"] <= 2 * nrhs, info
    xm = xm.reshape(nrhs, len(shifts), ctx.Vh, 3)
    # FP64 true residuals through the library and through the oracle operator
    # (the library certifies its own FP64 evaluation of |b - A x| <= res; the oracle's evaluation
    # rounds differently, by about 1e-16 |b| per component: ~3e-14 absolute here, 3e-4 of res)
    orc = oracle_mod.Oracle(dims)
    for r in range(nrhs):
        for i, s in enumerate(shifts):
            rr = bs[r] - orc.mdagm(u, xm[r, i], mass, s)
            assert np.linalg.norm(rr) <= res * (1 + 1e-3), (r, i, np.linalg.norm(rr))
    xf, _ = ctx.msolve_host(bs if nrhs > 1 else bs[0], shifts, res)
    xf = xf.reshape(nrhs, len(shifts), ctx.Vh, 3)
    assert rel_err(xm, xf) < 1e-8


def test_true_residuals_api(oracle_mod):
    from gpu_util import new_ctx, to_internal, internal_buffer
    import torch
    dims = (4, 6, 2, 10)
    mass = 0.1
    ctx = new_ctx(dims, mass=mass)
    u = F.random_links(dims, seed=141)
    ctx.set_gauge(u)
    b = F.random_spinor(dims, seed=142)
    xs = F.random_spinor(dims, seed=143, n=2)
    shifts = np.array([0.0, 0.5])
    bd = to_internal(ctx, rb.LINKS_F64_18, b)
    xd = to_internal(ctx, rb.LINKS_F64_18, xs)
    torch.cuda.synchronize()
    out = ctx.true_residuals(xd, bd, shifts)
    orc = oracle_mod.Oracle(dims)
    for i, s in enumerate(shifts):
        ref = np.linalg.norm(b - orc.mdagm(u, xs[i], mass, s))
        assert abs(out[0, i] - ref) <= 1e-12 * ref


def test_msolve_errors():
    from gpu_util import new_ctx
    dims = (4, 4, 4, 4)
    ctx = new_ctx(dims, mass=0.01)
    ctx.set_gauge(F.random_links(dims, seed=151))
    b = F.random_spinor(dims, seed=152)
    with pytest.raises(rb.RhmcError, match="-3"):
        ctx.msolve_host(b, [0.01], 1e-12, max_iter=3)
    bad = b.copy()
    bad[3, 1] = np.nan
    with pytest.raises(rb.RhmcError, match="-4"):
        ctx.msolve_host(bad, [0.01], 1e-10)
    with pytest.raises(rb.RhmcError, match="-1"):
        ctx.msolve_host(b, [-1.0], 1e-10)
    with pytest.raises(rb.RhmcError, match="-1"):
        ctx.msolve_host(b, np.ones(40), 1e-10)
    # the context stays usable after the failures
    x, info = ctx.msolve_host(b, [0.5], 1e-10)
    assert info["status"] == 0


def test_msolve_zero_rhs():
    from gpu_util import new_ctx
    dims = (4, 4, 4, 4)
    ctx = new_ctx(dims, mass=0.1)
    ctx.set_gauge(F.random_links(dims, seed=161))
    x, info = ctx.msolve_host(np.zeros((ctx.Vh, 3), np.complex128), [0.1, 1.0], 1e-10)
    assert info["status"] == 0
    assert not np.any(x)


@pytest.mark.parametrize("mode,fmt", [(rb.MSOLVE_FP64, rb.LINKS_F64_18), (rb.MSOLVE_MIXED, rb.LINKS_F64_12)])
def test_msolve_pole_set_per_rhs(mode, fmt, oracle_mod):
    """Right-hand sides batched with a pole set each (e.g. two fermion species): FP64 mode
    reproduces each RHS's own single-RHS solve bit for bit; the mixed mode meets the FP64 true
    residual of every system."""
    from gpu_util import new_ctx
    dims = (6, 4, 4, 8)
    mass = 0.05
    ctx = new_ctx(dims, mass=mass)
    u = F.random_links(dims, seed=151)
    ctx.set_gauge(u)
    bs = F.random_spinor(dims, seed=152, n=2)
    sets = np.stack([shifts_log(6, 1e-3, 5.0), shifts_log(6, 2e-2, 40.0)])
    res = 1e-10
    xb, info = ctx.msolve_host(bs, sets, res, mode=mode, fmt=fmt)
    assert info["status"] == 0, info
    orc = oracle_mod.Oracle(dims)
    for r in range(2):
        if mode == rb.MSOLVE_FP64:
            x1, _ = ctx.msolve_host(bs[r], sets[r], res)
            assert np.array_equal(x1, xb[r])
        for i, sg in enumerate(sets[r]):
            rr = bs[r] - orc.mdagm(u, xb[r, i], mass, sg)
            if mode == rb.MSOLVE_MIXED:  # certified by the library's own FP64 evaluation (see above)
                assert np.linalg.norm(rr) <= res * (1 + 1e-3), (r, i, np.linalg.norm(rr))
