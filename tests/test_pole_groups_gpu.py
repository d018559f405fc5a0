"""Pole groups (rhmc_driver_params.pole_group): the driver may solve an approximation's poles a
few at a time, using each group's shifted solutions (its share of the rational sum, force or
action) and dropping them before the next group, so that only one group's shifted vectors are
on the device.  The results are those of the all-poles solve up to the solver tolerance: both
solve every (M^dag M + sigma_i) x_i = b to residual 1e-12, so heatbath, action and force agree
to 1e-9 relative and a trajectory gives the same Delta H to 1e-7 and the same decision.  The
grouped run also holds less workspace memory (measured after releasing the workspaces).

Two species (N_f = 2 light + N_f = 1 heavier, two pseudofermions each) on the 4^4 fixture links,
with the fixture's degree-8 coefficients, in groups of 3 poles (3 + 3 + 2)."""
import json
import os

import numpy as np
import pytest

import rhmc_b200 as rb
from rhmc_b200 import fields as F
from conftest import rel_err

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
M_S = 0.2


def _run(pole_group):
    from gpu_util import new_ctx
    g = dict(np.load(os.path.join(HERE, "golden", "ref_t4.npz")))
    with open(os.path.join(HERE, "golden", "rational_coeffs.json")) as f:
        cf = json.load(f)["t4"]
    m = float(g["mass"])
    dims = tuple(g["dims"])
    b_l = tuple(g["bounds"])
    b_s = tuple(np.array(b_l) + M_S ** 2 - m ** 2)
    ctx = new_ctx(dims, mass=m, beta=float(g["beta"]))
    ctx.set_gauge(g["u"])
    ctx.driver_setup(no_flavours=2, no_ps=2, no_md=5, integrator=rb.INT_LEAPFROG, residue_md=1e-12,
                     residue_metro=1e-12, pole_group=pole_group)
    assert ctx.add_species(M_S, 1, 2) == 1
    phis = [F.random_spinor(dims, seed=2105, n=2), F.random_spinor(dims, seed=2106, n=2)]
    for s, b in enumerate((b_l, b_s)):
        ctx.select_species(s)
        for w, c in enumerate(cf):
            ctx.set_approx(w, c)
        ctx.set_eig_bounds(*b)
        ctx.set_phi(phis[s])
    ctx.workspace_release()
    ctx.first_inv_approx_calc(1e-12)
    chis = []
    for s in range(2):
        ctx.select_species(s)
        chis.append(ctx.get_chi())
    ctx.select_species(0)
    act = ctx.fermion_action()
    ctx.calc_ipdot_fermion()
    ip = ctx.get_ipdot()
    ws = ctx.workspace_bytes()
    # one trajectory from the same momenta and phi
    ctx.set_momenta(F.random_momenta(dims, seed=2107))
    for s in range(2):
        ctx.select_species(s)
        ctx.set_phi(phis[s])
    ctx.select_species(0)
    de, acc = ctx.update(0.5)
    plaq = ctx.plaquette()
    ctx.close()
    return chis, act, ip, ws, de, acc, plaq


def test_pole_groups_match_all_poles():
    c0, a0, i0, ws0, de0, acc0, pl0 = _run(0)
    c1, a1, i1, ws1, de1, acc1, pl1 = _run(3)
    for s in range(2):
        assert rel_err(c1[s], c0[s]) < 1e-9
    assert abs(a1 - a0) <= 1e-9 * abs(a0)
    assert rel_err(i1, i0) < 1e-9
    assert abs(de1 - de0) < 1e-7
    assert acc1 == acc0
    assert np.allclose(pl1, pl0, rtol=0, atol=1e-9)
    # the grouped solves keep 3 instead of 8 shifted solutions (and directions) per right-hand side
    assert ws1 < ws0


def test_pole_group_rejects_negative():
    from gpu_util import new_ctx
    ctx = new_ctx((4, 4, 4, 4))
    with pytest.raises(rb.RhmcError):
        ctx.driver_setup(pole_group=-1)


def test_driver_solver_stats():
    """rhmc_driver_solver_stats sums the driver's solves by kind: heatbath/action solves into one
    sum, force solves into the other, and resets on request."""
    from gpu_util import new_ctx
    g = dict(np.load(os.path.join(HERE, "golden", "ref_t4.npz")))
    with open(os.path.join(HERE, "golden", "rational_coeffs.json")) as f:
        cf = json.load(f)["t4"]
    ctx = new_ctx(tuple(g["dims"]), mass=float(g["mass"]), beta=float(g["beta"]))
    ctx.set_gauge(g["u"])
    ctx.driver_setup(no_flavours=2, no_ps=1, residue_md=1e-10, residue_metro=1e-12)
    for w, c in enumerate(cf):
        ctx.set_approx(w, c)
    ctx.set_eig_bounds(*tuple(g["bounds"]))
    ctx.set_phi(g["phi"])
    ctx.first_inv_approx_calc(1e-12)
    md, metro = ctx.driver_solver_stats(0), ctx.driver_solver_stats(1)
    assert md["iters_total"] == 0 and metro["iters_total"] > 0 and metro["seconds"] > 0
    ctx.calc_ipdot_fermion()
    md = ctx.driver_solver_stats(0, reset=True)
    assert md["iters_total"] > 0 and md["iters_max"] > 0
    assert ctx.driver_solver_stats(0)["iters_total"] == 0 and ctx.driver_solver_stats(1)["iters_total"] == 0
    with pytest.raises(rb.RhmcError):
        ctx.driver_solver_stats(2)
