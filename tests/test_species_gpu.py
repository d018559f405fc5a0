"""Fermion species (N_f = 2+1 style): a second species of mass m_s added to a context of mass m
must give exactly what a context of mass m_s gives for that species alone (its poles are
shifted by m_s^2 - m^2 on the context's M^dag M), and heatbath, action and force must sum over
the species.  Inputs: the 4^4 fixture links; both species use the fixture's rational
coefficients (the identities hold for any coefficients).  Solves at residual 1e-12, so the
tolerance is 1e-10 relative."""
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


def _data():
    g = dict(np.load(os.path.join(HERE, "golden", "ref_t4.npz")))
    with open(os.path.join(HERE, "golden", "rational_coeffs.json")) as f:
        cf = json.load(f)["t4"]
    return g, cf


def _ctx(g, cf, mass, no_flavours, bounds):
    from gpu_util import new_ctx
    ctx = new_ctx(tuple(g["dims"]), mass=mass, beta=float(g["beta"]))
    ctx.set_gauge(g["u"])
    ctx.driver_setup(no_flavours=no_flavours, no_ps=1, residue_md=1e-12, residue_metro=1e-12)
    for w, c in enumerate(cf):
        ctx.set_approx(w, c)
    ctx.set_eig_bounds(*bounds)
    return ctx


def _contexts():
    g, cf = _data()
    m = float(g["mass"])
    b_l = tuple(g["bounds"])
    b_s = tuple(np.array(b_l) + M_S ** 2 - m ** 2)
    light = _ctx(g, cf, m, 2, b_l)
    strange = _ctx(g, cf, M_S, 1, b_s)
    both = _ctx(g, cf, m, 2, b_l)
    s = both.add_species(M_S, 1, 1)
    assert s == 1
    both.select_species(s)
    for w, c in enumerate(cf):
        both.set_approx(w, c)
    both.set_eig_bounds(*b_s)
    return g, light, strange, both


def test_species_heatbath_action_force():
    g, light, strange, both = _contexts()
    phi_l = g["phi"]
    phi_s = F.random_spinor(tuple(g["dims"]), seed=2003, n=1)
    light.set_phi(phi_l)
    strange.set_phi(phi_s)
    both.select_species(0)
    both.set_phi(phi_l)
    both.select_species(1)
    both.set_phi(phi_s)
    for c in (light, strange, both):
        c.first_inv_approx_calc(1e-12)
    assert rel_err(both.get_chi(), strange.get_chi()) < 1e-10
    both.select_species(0)
    assert rel_err(both.get_chi(), light.get_chi()) < 1e-10
    # action and force of the md approximation sum over the species
    s_l, s_s, s_b = light.fermion_action(), strange.fermion_action(), both.fermion_action()
    assert abs(s_b - (s_l + s_s)) <= 1e-10 * abs(s_b)
    for c in (light, strange, both):
        c.calc_ipdot_fermion()
    ip = light.get_ipdot() + strange.get_ipdot()
    assert rel_err(both.get_ipdot(), ip) < 1e-10


def test_species_errors():
    g, light, strange, both = _contexts()
    with pytest.raises(rb.RhmcError):
        light.add_species(0.05, 1, 1)  # below the context mass
    with pytest.raises(rb.RhmcError):
        both.select_species(2)


def test_single_rhs_matches_batched():
    """The driver's single_rhs option (every pseudofermion in its own solve, as the reference's
    loop over pseudofermions) and the default batched solve give the same heatbath, action and
    force: in FP64 mode each right-hand side of a batched solve follows its own recurrences with
    launch-shape-independent reductions."""
    g, cf = _data()
    m = float(g["mass"])
    dims = tuple(g["dims"])
    b_l = tuple(g["bounds"])
    b_s = tuple(np.array(b_l) + M_S ** 2 - m ** 2)
    phis = [F.random_spinor(dims, seed=2005, n=2), F.random_spinor(dims, seed=2006, n=2)]
    out = []
    for single in (0, 1):
        from gpu_util import new_ctx
        ctx = new_ctx(dims, mass=m, beta=float(g["beta"]))
        ctx.set_gauge(g["u"])
        ctx.driver_setup(no_flavours=2, no_ps=2, residue_md=1e-12, residue_metro=1e-12, single_rhs=single)
        assert ctx.add_species(M_S, 1, 2) == 1
        for s, b in enumerate((b_l, b_s)):
            ctx.select_species(s)
            for w, c in enumerate(cf):
                ctx.set_approx(w, c)
            ctx.set_eig_bounds(*b)
            ctx.set_phi(phis[s])
        ctx.first_inv_approx_calc(1e-12)
        chis = []
        for s in range(2):
            ctx.select_species(s)
            chis.append(ctx.get_chi())
        ctx.select_species(0)
        act = ctx.fermion_action()
        ctx.calc_ipdot_fermion()
        out.append((chis, act, ctx.get_ipdot()))
    (c0, a0, i0), (c1, a1, i1) = out
    for s in range(2):
        assert rel_err(c1[s], c0[s]) < 1e-14
    assert abs(a1 - a0) <= 1e-14 * abs(a0)
    assert rel_err(i1, i0) < 1e-14
