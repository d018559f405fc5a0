"""Forces, updates and the molecular-dynamics driver on the B200 against fixtures recorded from
the reference's own CPU code (tests/golden/make_golden.py) and against the oracle.

Tolerances (relative L2 unless stated): gauge force 1e-13, heatbath chi and fermion force 1e-11
(multi-shift solves at 1e-10 / 1e-8 in between), momentum update 1e-14, link update 1e-13;
trajectories: identical accept/reject, |Delta S - Delta S_ref| <= 1e-6 max(1, |Delta S_ref|),
plaquette within 1e-9 (FP64 rounding differences grow along a chaotic MD trajectory).
"""
import json
import os

import numpy as np
import pytest

import rhmc_b200 as rb
from rhmc_b200 import fields as F
from conftest import rel_err

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TAGS = ["t4", "a6448"]


def load(tag):
    return dict(np.load(os.path.join(HERE, "golden", "ref_%s.npz" % tag)))


def coeffs(tag):
    with open(os.path.join(HERE, "golden", "rational_coeffs.json")) as f:
        return json.load(f)[tag]


def setup(tag, integrator=rb.INT_2MN):
    from gpu_util import new_ctx
    g = load(tag)
    ctx = new_ctx(tuple(g["dims"]), mass=float(g["mass"]), beta=float(g["beta"]))
    ctx.set_gauge(g["u"])
    ctx.driver_setup(no_flavours=int(g["no_flavours"]), no_ps=int(g["no_ps"]), no_md=int(g["no_md"]),
                     gauge_scale=int(g["gauge_scale"]), integrator=integrator, residue_metro=float(g["residue_metro"]),
                     residue_md=float(g["residue_md"]))
    for w, c in enumerate(coeffs(tag)):
        ctx.set_approx(w, c)
    ctx.set_eig_bounds(*g["bounds"])
    return ctx, g


@pytest.mark.parametrize("tag", TAGS)
def test_gauge_force_vs_reference(tag):
    ctx, g = setup(tag)
    ctx.gauge_force(0)
    assert rel_err(ctx.get_ipdot(), g["ipdot_gauge"]) < 1e-13


@pytest.mark.parametrize("tag", TAGS)
def test_heatbath_and_fermion_force_vs_reference(tag):
    ctx, g = setup(tag)
    ctx.set_phi(g["phi"])
    ctx.first_inv_approx_calc(1e-10)
    assert rel_err(ctx.get_chi(), g["chi"]) < 1e-11
    ctx.set_chi(g["chi"])
    ctx.calc_ipdot_fermion()
    assert rel_err(ctx.get_ipdot(), g["ipdot_fermion"]) < 1e-11
    ctx.calc_ipdot()
    assert rel_err(ctx.get_ipdot(), g["ipdot_full"]) < 1e-11


def test_updates_and_plaquette_vs_reference():
    ctx, g = setup("t4")
    s, t = ctx.plaquette()
    assert abs(s - g["plaq"][0]) < 1e-13 and abs(t - g["plaq"][1]) < 1e-13
    ctx.set_momenta(g["P"])
    ctx.set_ipdot(g["ipdot_full"])
    ctx.mom_update(-0.05)
    assert rel_err(ctx.get_momenta(), g["P_after"]) < 1e-14
    ctx.link_update(0.05)
    assert rel_err(ctx.get_gauge(), g["u_after"]) < 1e-13


@pytest.mark.parametrize("tag", TAGS)
@pytest.mark.parametrize("integ", [rb.INT_2MN, rb.INT_MULTISTEP_2MN, rb.INT_MULTISTEP_4MN, rb.INT_LEAPFROG])
def test_trajectory_vs_reference(tag, integ):
    ctx, g = setup(tag, integ)
    ctx.set_momenta(g["P"])
    ctx.set_phi(g["phi"])
    de, acc = ctx.update(float(g["uniform"]))
    de_ref = float(g["traj%d_de" % integ])
    assert acc == int(g["traj%d_acc" % integ])
    assert abs(de - de_ref) <= 1e-6 * max(1.0, abs(de_ref)), (de, de_ref)
    s, t = ctx.plaquette()
    ps, pt = g["traj%d_plaq" % integ]
    assert abs(s - ps) < 1e-9 and abs(t - pt) < 1e-9
    if integ == 0:
        assert rel_err(ctx.get_gauge(), g["traj0_u"]) < 1e-9


@pytest.mark.parametrize("dims", [(4, 6, 2, 10), (6, 4, 4, 8)])
def test_forces_vs_oracle(dims):
    """Other lattice shapes: gauge and fermion force against the C restatement."""
    import oracle
    import torch
    from gpu_util import new_ctx, to_internal
    beta, mass = 5.6, 0.07
    ctx = new_ctx(dims, mass=mass, beta=beta)
    u = F.random_links(dims, seed=501)
    ctx.set_gauge(u)
    orc = oracle.Oracle(dims)
    ctx.gauge_force(0)
    assert rel_err(ctx.get_ipdot(), orc.ipdot_gauge(u, beta)) < 1e-13
    xs = F.random_spinor(dims, seed=502, n=6)  # 2 rhs x 3 shifts
    a = np.array([0.3, -0.7, 1.1])
    xd = to_internal(ctx, rb.LINKS_F64_18, xs)
    torch.cuda.synchronize()
    ctx.fermion_force(xd, a, nrhs=2, add=1)
    buf = orc.ipdot_gauge_init(u, beta)
    orc.fermion_force_accum(buf, u, xs[:3], a)
    orc.fermion_force_accum(buf, u, xs[3:], a)
    assert rel_err(ctx.get_ipdot(), orc.u_times_ta(u, buf)) < 1e-12


def test_actions_vs_oracle():
    import oracle
    dims = (4, 6, 2, 10)
    ctx = rb.Context(dims, mass=0.1, beta=5.5)
    u = F.random_links(dims, seed=511)
    P = F.random_momenta(dims, seed=512)
    ctx.set_gauge(u)
    ctx.set_momenta(P)
    orc = oracle.Oracle(dims)
    assert abs(ctx.gauge_action() - orc.gauge_action(u, 5.5)) < 1e-12 * abs(orc.gauge_action(u, 5.5))
    assert abs(ctx.momentum_action() - orc.momentum_action(P)) < 1e-12 * orc.momentum_action(P)
    s, t = ctx.plaquette()
    so, to = orc.plaquette(u)
    assert abs(s - so) < 1e-14 and abs(t - to) < 1e-14


def test_driver_errors_and_reject_restores_links():
    from gpu_util import new_ctx
    dims = (4, 4, 4, 4)
    ctx = new_ctx(dims)
    with pytest.raises(rb.RhmcError, match="-5"):
        ctx.update_nometro()
    ctx2, g = setup("t4", rb.INT_LEAPFROG)  # this trajectory is rejected by the reference
    ctx2.set_momenta(g["P"])
    ctx2.set_phi(g["phi"])
    de, acc = ctx2.update(float(g["uniform"]))
    assert acc == 0
    assert np.array_equal(ctx2.get_gauge(), g["u"])


@pytest.mark.parametrize("auto", [1, 2])
def test_driver_auto_bounds(auto):
    """auto_bounds: the driver computes lambda_min/max of M^dag M by FP64 power iterations at the
    start of every trajectory (as findminmax does at every rescaling); with 2 lambda_min = m^2.
    The bounds must enclose the spectrum the power iterations of the legacy entry points give and
    a trajectory must run with them."""
    from gpu_util import new_ctx
    g = load("t4")
    mass = float(g["mass"])
    ctx = new_ctx(tuple(g["dims"]), mass=mass, beta=float(g["beta"]))
    ctx.set_gauge(g["u"])
    ctx.driver_setup(no_flavours=2, no_ps=1, no_md=4, integrator=rb.INT_LEAPFROG, auto_bounds=auto)
    for w, c in enumerate(coeffs("t4")):
        ctx.set_approx(w, c)
    # the bounds belong to the trajectory's starting configuration
    ref_max = ctx.find_max(F.random_spinor(tuple(g["dims"]), seed=77))
    ctx.set_momenta(g["P"])
    ctx.set_phi(g["phi"])
    de, acc = ctx.update(0.5)
    assert np.isfinite(de)
    mn, mx = ctx.eig_bounds()
    # two power iterations from different starts; the 5e-4 stop on the relative change of the norm
    # leaves each a little below lambda_max when the top eigenvalues are close (the rescaling's
    # factor 1.05 covers that, as in the reference)
    assert abs(mx - ref_max) <= 2e-2 * ref_max
    if auto == 2:
        assert mn == mass * mass
    else:
        assert mass * mass * 0.999 < mn < mx
