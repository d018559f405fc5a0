"""The reference's extern "C" GPU entry points (include/rhmc_legacy.h) driven as the reference's
host code drives them (gpu.cc, cu_inverter.cc, rationalapprox.cc, fermionforce.cc, ipdot.cc,
momenta.cc, findminmax.cc), on host buffers in the packer formats, against fixtures recorded
from the reference's CPU code.

Tolerances: links and chi travel as float hi+lo pairs (~1e-14 relative); ipdot and momenta
travel as single floats and the force numerators are floats in this interface, so those are
compared at 2e-7 / 1e-6 relative.
"""
import json
import os

import numpy as np
import pytest

import rhmc_b200 as rb
from rhmc_b200 import fields as F
from rhmc_b200 import rational as R
from conftest import rel_err
import legacy_pack as LP

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))


def rescaled(g, which, approx):
    mx = float(g["bounds"][1]) * 1.05
    nf, nps = int(g["no_flavours"]), int(g["no_ps"])
    ex = nf / 8.0 / nps if which == 0 else -nf / 4.0 / nps
    return R.rescale(approx, mx, ex)


@pytest.mark.parametrize("tag", ["t4", "a6448"])
def test_legacy_entry_points_vs_reference(tag):
    g = dict(np.load(os.path.join(HERE, "golden", "ref_%s.npz" % tag)))
    with open(os.path.join(HERE, "golden", "rational_coeffs.json")) as f:
        cf = json.load(f)[tag]
    dims = tuple(int(d) for d in g["dims"])
    V = int(np.prod(dims))
    Vh = V // 2
    nps = int(g["no_ps"])
    order = max(len(c["a"]) for c in cf)
    bufs = {
        "gauge_field_packed": LP.pack_gauge(g["u"]),
        "chi_packed": LP.pack_multifermion(g["phi"]),  # gpu_init1 packs fermion_phi (gpu.cc:17-23)
        "simple_fermion_packed": LP.pack_fermion_d(g["x"]),
        "ipdot_packed": LP.pack_tamatrix(np.zeros((4 * V, 3, 3), np.complex128)),
        "momenta_packed": LP.pack_thmatrix(g["P"]),
        "shift_table": F.neighbour_table(dims),
        "eta": F.eta_phases(dims),
    }
    leg = rb.Legacy(dims, float(g["mass"]), float(g["beta"]), nps, order, 20000, bufs)
    leg.cuda_init0()
    leg.cuda_init1()
    ctx = rb.Context.wrap(leg.context_handle(), dims, float(g["mass"]), float(g["beta"]))
    assert rel_err(ctx.get_gauge(), g["u"]) < 1e-13
    # first_inv_approx_calc on the GPU path (rationalapprox.cc:278-291)
    first = rescaled(g, 0, cf[0])
    for ps in range(nps):
        assert leg.shifted_inverter(1e-10, first["b"], ps) > 0
    leg.sol_sum(first["a0"], first["a"])
    chi = LP.unpack_multifermion(bufs["chi_packed"], nps, Vh)
    assert rel_err(chi, g["chi"]) < 1e-12
    # calc_ipdot on the GPU path (ipdot.cc:160-163 -> fermionforce.cc:31-45)
    md = rescaled(g, 1, cf[1])
    for ps in range(nps):
        leg.shifted_inverter(float(g["residue_md"]), md["b"], ps)
    leg.fermion_force(np.array(md["a"], np.float32))
    leg.cuda_gauge_deriv(1)
    leg.cuda_end()
    ip = LP.unpack_alg(bufs["ipdot_packed"], V, True)
    assert rel_err(ip, g["ipdot_full"]) < 2e-7
    # momenta_sum_multiply on the GPU path (momenta.cc:93-95), with the fixture's ipdot
    ctx.set_ipdot(g["ipdot_full"])
    leg.cuda_put_momenta()
    leg.cuda_momenta_sum_multiply(np.float32(-0.05))
    leg.cuda_get_momenta()
    P = LP.unpack_alg(bufs["momenta_packed"], V, False)
    assert rel_err(P, g["P_after"]) < 1e-6
    # gauge links back through the packed format
    leg.cuda_get_conf()
    rows = LP.unpack_gauge_rows01(bufs["gauge_field_packed"], V)
    assert rel_err(rows, g["u"][:, :2, :]) < 1e-13


def test_legacy_power_iteration_matches_oracle():
    import oracle
    g = dict(np.load(os.path.join(HERE, "golden", "ref_t4.npz")))
    dims = tuple(int(d) for d in g["dims"])
    V = int(np.prod(dims))
    mass = float(g["mass"])
    # findminmax packs the start vector single precision into the first 6*Vh floats
    # (findminmax.cc:161); the rest of the buffer holds another vector, which must be ignored
    sfp = LP.pack_fermion_d(g["phi"][0])
    sfp[:6 * (V // 2)] = LP.pack_fermion(g["x"])
    bufs = {"gauge_field_packed": LP.pack_gauge(g["u"]), "chi_packed": LP.pack_multifermion(g["phi"]),
            "simple_fermion_packed": sfp,
            "ipdot_packed": LP.pack_tamatrix(np.zeros((4 * V, 3, 3), np.complex128)),
            "momenta_packed": LP.pack_thmatrix(g["P"])}
    leg = rb.Legacy(dims, mass, float(g["beta"]), 1, 8, 20000, bufs)
    leg.cuda_init0()
    leg.cuda_init1()
    mx = leg.find_max()
    mn = leg.find_min(mx)
    # the same power iterations in FP64 with the oracle operator
    orc = oracle.Oracle(dims)
    hi = LP.pack_fermion(g["x"]).astype(np.float64)
    start = hi[0::2].reshape(3, V // 2).T + 1j * hi[1::2].reshape(3, V // 2).T

    def power(shift_max, for_min):
        p = start.copy()
        nrm = np.linalg.norm(p)
        while True:
            p = p / nrm
            old = nrm
            q = orc.mdagm(g["u"], p, mass)
            p = shift_max * p - q if for_min else q
            nrm = np.linalg.norm(p)
            rel = abs(old - nrm) / (abs(shift_max - nrm) if for_min else nrm)
            if rel <= 5e-4:
                return shift_max - nrm if for_min else nrm

    assert abs(mx - power(0.0, False)) < 1e-9 * mx
    assert abs(mn - power(mx, True)) < 1e-9 * mx
    assert mass ** 2 * 0.999 < mn < mx < 16.0 + mass ** 2
    # single-precision inverter (the reference's SP path) runs and reports its iterations
    assert leg.shifted_inverter(1e-4, [0.01, 0.1, 1.0], 0, double=False) > 0
