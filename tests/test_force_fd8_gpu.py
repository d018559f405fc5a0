"""The fermion force against the 2-point central difference of S_f with the stencil of the
fermion-force check configuration (eps = 1e-5, 8 random su(3) directions, seed 5005, on 16
random links, seed 6006), here on an 8^4 lattice with am = 0.05 and a degree-12 near-minimax
approximation of x^(-1/2): |FD - Re(i Tr(Q ipdot_l))| <= 1e-8 |Q| |ipdot_l| for every pair.

S(+eps) - S(-eps) is not taken as the difference of two summed actions (which loses digits to
cancellation) but evaluated exactly by the second resolvent identity,
    S(+) - S(-) = sum_i a_i Re<x_i(+), (A(-) - A(+)) x_i(-)>,   A(+-) = M^dag M(+-) + b_i,
with x_i(+-) = A(+-)^-1 chi solved in FP64 to a true residual of 1e-12 (certified); the sigma_i
cancel in A(-) - A(+), which is non-zero only next to the perturbed link.
"""
import numpy as np
import pytest
from scipy.linalg import expm

import rhmc_b200 as rb
from rhmc_b200 import fields as F
from rhmc_b200 import rational as R

pytestmark = pytest.mark.gpu


def test_fermion_force_fd_resolvent_8x4():
    import torch
    from gpu_util import new_ctx
    dims, mass, deg = (8, 8, 8, 8), 0.05, 12
    V = int(np.prod(dims))
    Vh = V // 2
    ctx = new_ctx(dims, mass=mass, beta=5.5)
    u = F.random_links(dims, seed=1001, kind="near1")
    ctx.set_gauge(u)
    lmin, lmax = mass * mass, 16.0 + mass * mass
    eps = lmin / (1.05 * lmax)
    approx = [R.rational_power(0.25, deg, eps), R.rational_power(-0.5, deg, eps), R.rational_power(-0.5, deg, eps)]
    assert approx[1]["max_rel_err"] < 1e-5
    ctx.driver_setup(no_flavours=2, no_ps=1, residue_md=1e-12, residue_metro=1e-12)
    for w, c in enumerate(approx):
        ctx.set_approx(w, c)
    ctx.set_eig_bounds(lmin, lmax)
    chi_host = F.random_spinor(dims, seed=2002, n=1)
    ctx.set_chi(chi_host)
    ctx.calc_ipdot_fermion()
    ip = ctx.get_ipdot()
    md = R.rescale(approx[1], 1.05 * lmax, -0.5)  # rationalapprox.cc:206-214: N_f/(4 N_ps) = 1/2
    shifts, a = np.array(md["b"]), np.array(md["a"])
    dev = torch.device("cuda")
    chi = torch.zeros(6 * Vh, dtype=torch.float64, device=dev)
    ctx.spinor_to_internal(rb.LINKS_F64_18, chi, chi_host[0])
    x = {s: torch.zeros(deg * 6 * Vh, dtype=torch.float64, device=dev) for s in (-1, 1)}
    w1 = torch.zeros(deg * 6 * Vh, dtype=torch.float64, device=dev)
    w2 = torch.zeros_like(w1)
    ta = torch.as_tensor(a, device=dev)
    links = np.random.Generator(np.random.Philox(6006)).choice(4 * V, size=16, replace=False)
    Qs = F.random_algebra(8, np.random.Generator(np.random.Philox(5005)))
    h = 1e-5
    u_dev = torch.from_numpy(u).to(dev)
    worst = 0.0
    for l in links:
        ul = u[l].copy()
        for Q in Qs:
            for sign in (-1, 1):
                u_dev[l] = torch.from_numpy(expm(1j * sign * h * Q) @ ul).to(dev)
                ctx.set_gauge(u_dev)
                info = ctx.msolve(x[sign], chi, shifts, 1e-12, certify=1)
                assert info["status"] == 0
                # M^dag M x_i(-) at this configuration (the shifts cancel in the difference)
                ctx.mdagm(rb.LINKS_F64_18, w1 if sign < 0 else w2, x[-1], 0.0, deg)
            torch.cuda.synchronize()
            d = (x[1].view(deg, 6 * Vh) * (w1 - w2).view(deg, 6 * Vh)).sum(1)
            fd = float((ta * d).sum()) / (2 * h)
            exact = float((1j * np.trace(Q @ ip[l])).real)
            rel = abs(fd - exact) / (np.linalg.norm(Q) * np.linalg.norm(ip[l]))
            worst = max(worst, rel)
            assert rel <= 1e-8, (int(l), fd, exact, rel)
        u_dev[l] = torch.from_numpy(ul).to(dev)
    ctx.set_gauge(u)
    print("max relative error %.3g over %d pairs" % (worst, 16 * 8))
