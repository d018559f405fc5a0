"""The hand-written fermion force (the adjoint of the pseudofermion action) and the gauge force
against central finite differences of their actions, along random su(3) directions on random
links: with U_l -> exp(i t Q) U_l, dS/dt at t = 0 must equal Re(i Tr(Q ipdot_l)).

S_f is evaluated with FP64 solves at residual 1e-13 (its error is quadratic in the CG error).
Errors are relative to |Q| |ipdot_l| (Frobenius norms), the bound of the projection: a 4-point
central difference at h = 1e-4 must agree to 1e-8 (round-off and truncation are both below
that), the plain 2-point central difference at eps = 1e-5 to 1e-7.
"""
import json
import os

import numpy as np
import pytest
from scipy.linalg import expm

import rhmc_b200 as rb
from rhmc_b200 import fields as F

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def _setup(two_species=False, minimax=False):
    from gpu_util import new_ctx
    g = dict(np.load(os.path.join(HERE, "golden", "ref_t4.npz")))
    with open(os.path.join(HERE, "golden", "rational_coeffs.json")) as f:
        cf = json.load(f)["t4"]
    if minimax:  # near-minimax type (n, n) coefficients: a0 != 0 in the action's approximation
        from rhmc_b200 import rational as R
        cf = [R.rational_power(c["power"], len(c["a"]), c["min_eps"], method="minimax") for c in cf]
    m = float(g["mass"])
    ctx = new_ctx(tuple(g["dims"]), mass=m, beta=float(g["beta"]))
    ctx.driver_setup(no_flavours=2, no_ps=1, residue_md=1e-13, residue_metro=1e-13)
    for w, c in enumerate(cf):
        ctx.set_approx(w, c)
    ctx.set_eig_bounds(*g["bounds"])
    ctx.set_chi(g["chi"])
    if two_species:  # a heavier species (mass 0.25, one flavour) with its own pseudofermion
        s = ctx.add_species(0.25, 1, 1)
        ctx.select_species(s)
        for w, c in enumerate(cf):
            ctx.set_approx(w, c)
        ctx.set_eig_bounds(*(np.array(g["bounds"]) + 0.25 ** 2 - m ** 2))
        ctx.set_chi(F.random_spinor(tuple(g["dims"]), seed=2003, n=1))
    return ctx, g


def _fd(ctx, u, l, Q, action, h, four_point):
    def S(t):
        v = u.copy()
        v[l] = expm(1j * t * Q) @ v[l]
        ctx.set_gauge(v)
        return action()
    if four_point:
        return (8 * (S(h) - S(-h)) - (S(2 * h) - S(-2 * h))) / (12 * h)
    return (S(h) - S(-h)) / (2 * h)


@pytest.mark.parametrize("part", ["fermion", "fermion_2species", "fermion_minimax", "gauge"])
def test_force_is_the_derivative_of_its_action(part):
    ctx, g = _setup(part == "fermion_2species", part == "fermion_minimax")
    u = g["u"]
    rng = np.random.Generator(np.random.Philox(6006))
    links = rng.choice(u.shape[0], size=4, replace=False)
    Qs = F.random_algebra(4, np.random.Generator(np.random.Philox(5005)))
    ctx.set_gauge(u)
    if part.startswith("fermion"):
        ctx.calc_ipdot_fermion()
        action = ctx.fermion_action
    else:
        ctx.gauge_force(0)
        action = ctx.gauge_action
    ip = ctx.get_ipdot()
    for l in links:
        for Q in Qs:
            exact = (1j * np.trace(Q @ ip[l])).real
            scale = np.linalg.norm(Q) * np.linalg.norm(ip[l])
            fd4 = _fd(ctx, u, l, Q, action, 1e-4, True)
            fd2 = _fd(ctx, u, l, Q, action, 1e-5, False)
            assert abs(fd4 - exact) <= 1e-8 * scale, (part, l, fd4, exact)
            assert abs(fd2 - exact) <= 1e-7 * scale, (part, l, fd2, exact)
    ctx.set_gauge(u)
