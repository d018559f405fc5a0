"""The t-slab decomposition's local compute on the GPU (one GPU here): the library's site-range
Dslash (rhmc_dslash_sites) on each rank's extended lattice -- interior output sites only,
parity shifted by the ghost slice, ghost links and spinor faces as the exchange delivers them --
gives each rank's slice of the single-domain Dslash, for two and four ranks emulated one after
the other; and the whole decomposed operator and multi-shift CG with one rank (the faces are its
own slices) equal the single-domain library results.  The communication between GPUs (NCCL
send/recv of faces, all-reduce of the scalars) is covered by the gloo test on CPU; several GPUs
are not available in this pool."""
import numpy as np
import pytest

import rhmc_b200 as rb
from rhmc_b200 import domain as D
from rhmc_b200 import fields as F
from conftest import rel_err

pytestmark = pytest.mark.gpu
DIMS = (6, 4, 4, 8)


@pytest.mark.parametrize("world", [2, 4])
def test_site_range_dslash_per_rank(world):
    import torch
    from gpu_util import new_ctx
    u = F.random_links(DIMS, seed=1001)
    x = F.random_spinor(DIMS, seed=2002)
    ctx = new_ctx(DIMS)
    ctx.set_gauge(u)
    full = {p: np.zeros_like(x) for p in (0, 1)}
    for p in (0, 1):
        ctx.dslash_host(p, full[p], x)
    for r in range(world):
        slab = D.TSlab(DIMS, r, world)
        ce = rb.Context(slab.dims_ext, mass=0.1, ferm_temp_bc=1)
        ce.set_stream(torch.cuda.current_stream().cuda_stream)
        ce.set_gauge(slab.links_from_global(u))
        xin = torch.from_numpy(D.spinor_ext_from_global(slab, x)).cuda()
        a, b = slab.local_slice()
        i0, i1 = slab.interior()
        for p in (0, 1):
            out = torch.zeros_like(xin)
            D.library_dslash(ce, slab)(slab.ext_parity(p), out, xin)
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert rel_err(got[i0:i1], full[p][a:b]) < 1e-14, (r, p)
            assert not np.any(got[:i0]) and not np.any(got[i1:])  # only the interior is written
        ce.close()


def test_site_range_rejects_bad_ranges():
    from gpu_util import new_ctx
    import torch
    ctx = new_ctx(DIMS)
    ctx.set_gauge(F.random_links(DIMS, seed=1))
    buf = torch.zeros((ctx.Vh, 3), dtype=torch.complex128, device="cuda")
    for lo, n in ((-1, 4), (0, 0), (ctx.Vh - 2, 4)):
        with pytest.raises(rb.RhmcError, match="-1"):
            ctx.dslash_sites(0, buf, buf, lo, n)


def test_single_rank_decomposed_solver_matches_library():
    import torch
    from gpu_util import new_ctx
    mass = 0.1
    u = F.random_links(DIMS, seed=1001)
    b = F.random_spinor(DIMS, seed=2002)
    shifts = [0.003, 0.05, 0.7, 9.0]
    ctx = new_ctx(DIMS, mass=mass)
    ctx.set_gauge(u)
    xr, info = ctx.msolve_host(b, shifts, 1e-10)
    slab = D.TSlab(DIMS, 0, 1)
    ce = rb.Context(slab.dims_ext, mass=mass, ferm_temp_bc=1)
    ce.set_stream(torch.cuda.current_stream().cuda_stream)
    ce.set_gauge(slab.links_from_global(u))
    op = D.DDOperator(slab, mass, D.library_dslash(ce, slab))
    bl = torch.from_numpy(b).cuda()
    got = op.mdagm(bl, 0.5).cpu().numpy()
    from gpu_util import to_internal, from_internal, internal_buffer
    buf = internal_buffer(ctx, rb.LINKS_F64_18)
    ctx.mdagm(rb.LINKS_F64_18, buf, to_internal(ctx, rb.LINKS_F64_18, b), 0.5)
    ref = from_internal(ctx, rb.LINKS_F64_18, buf)
    assert rel_err(got, ref) < 1e-14
    # the library's FP64 solver also stops once every shift is frozen (the GPU solver's rule)
    xs, it = D.multishift_cg(op, bl, shifts, 1e-10, stop_on_frozen=True)
    assert abs(it - info["iters"][0]) <= 1
    for i in range(len(shifts)):
        assert rel_err(xs[i].cpu().numpy(), xr[i]) < 1e-9
    ce.close()
