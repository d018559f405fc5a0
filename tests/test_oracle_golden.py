"""The oracle's C restatement (oracle/rhmc_oracle.c) against fixtures recorded from the
reference's own CPU code (tests/golden/make_golden.py): pins the oracle before it is used as
the checker of the CUDA path.  CPU only."""
import json
import os

import numpy as np
import pytest

from conftest import rel_err
from rhmc_b200 import rational as R

HERE = os.path.dirname(os.path.abspath(__file__))
TAGS = ["t4", "a6448"]


def load(tag):
    return dict(np.load(os.path.join(HERE, "golden", "ref_%s.npz" % tag)))


def coeffs(tag):
    with open(os.path.join(HERE, "golden", "rational_coeffs.json")) as f:
        return json.load(f)[tag]


@pytest.fixture(scope="module")
def orc_mod():
    import oracle
    return oracle


def rescaled(g, which, approx):
    mx = float(g["bounds"][1]) * 1.05
    nf, nps = int(g["no_flavours"]), int(g["no_ps"])
    ex = nf / 8.0 / nps if which == 0 else -nf / 4.0 / nps
    return R.rescale(approx, mx, ex)


@pytest.mark.parametrize("tag", TAGS)
def test_tables_and_dslash_bit_exact(tag, orc_mod):
    g = load(tag)
    orc = orc_mod.Oracle(tuple(g["dims"]))
    t, e = orc.tables()
    assert np.array_equal(t, g["table"])
    assert np.array_equal(e, g["eta"])
    assert np.array_equal(orc.doe(g["u"], g["x"]), g["doe"])
    assert np.array_equal(orc.deo(g["u"], g["x"]), g["deo"])


@pytest.mark.parametrize("tag", TAGS)
def test_msolve(tag, orc_mod):
    g = load(tag)
    orc = orc_mod.Oracle(tuple(g["dims"]))
    x, it = orc.msolve(g["u"], g["x"], float(g["mass"]), g["ms_shifts"], 1e-10)
    assert rel_err(x, g["ms_x"]) < 1e-13


@pytest.mark.parametrize("tag", TAGS)
def test_heatbath_and_forces(tag, orc_mod):
    g = load(tag)
    orc = orc_mod.Oracle(tuple(g["dims"]))
    u, mass, beta = g["u"], float(g["mass"]), float(g["beta"])
    cf = coeffs(tag)
    # chi = r_first(M^dag M) phi per pseudofermion
    first = rescaled(g, 0, cf[0])
    chi = []
    for phi in g["phi"]:
        xs, _ = orc.msolve(u, phi, mass, first["b"], 1e-10)
        chi.append(orc.rational_sum(phi, xs, first["a0"], first["a"]))
    chi = np.array(chi)
    assert rel_err(chi, g["chi"]) < 1e-12
    # gauge force
    assert rel_err(orc.ipdot_gauge(u, beta), g["ipdot_gauge"]) < 1e-13
    # fermion force from the md approximation
    md = rescaled(g, 1, cf[1])
    F = np.zeros((u.shape[0], 3, 3), np.complex128)
    res_md = float(g["residue_md"])
    for c in g["chi"]:
        xs, _ = orc.msolve(u, c, mass, md["b"], res_md)
        orc.fermion_force_accum(F, u, xs, md["a"])
    assert rel_err(orc.u_times_ta(u, F), g["ipdot_fermion"]) < 1e-12
    # full: beta/3 staples + fermion outer products, then TA(U .)
    buf = orc.ipdot_gauge_init(u, beta)
    for c in g["chi"]:
        xs, _ = orc.msolve(u, c, mass, md["b"], res_md)
        orc.fermion_force_accum(buf, u, xs, md["a"])
    assert rel_err(orc.u_times_ta(u, buf), g["ipdot_full"]) < 1e-12


def test_updates_and_plaquette(orc_mod):
    g = load("t4")
    orc = orc_mod.Oracle(tuple(g["dims"]))
    P = g["P"].copy()
    orc.mom_update(P, g["ipdot_full"], -0.05)
    assert rel_err(P, g["P_after"]) < 1e-15
    u = g["u"].copy()
    orc.link_update(u, g["P_after"], 0.05)
    assert rel_err(u, g["u_after"]) < 1e-14
    s, t = orc.plaquette(g["u"])
    assert abs(s - g["plaq"][0]) < 1e-14 and abs(t - g["plaq"][1]) < 1e-14


def test_rational_coefficients_quality():
    """The committed coefficients approximate their powers on [eps, 1] (quality, not parity)."""
    with open(os.path.join(HERE, "golden", "rational_coeffs.json")) as f:
        allc = json.load(f)
    for tag, cs in allc.items():
        for c in cs:
            x = np.geomspace(c["min_eps"], 1.0, 500)
            r = c["a0"] + (np.array(c["a"])[None, :] / (x[:, None] + np.array(c["b"])[None, :])).sum(1)
            err = np.max(np.abs(r / x ** c["power"] - 1))
            assert err < 1e-3, (tag, c["power"], err)
            assert min(c["b"]) > 0


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libref_t4.so")),
                    reason="reference harness not built")
def test_reference_harness_reproduces_fixture(orc_mod):
    """Re-run the reference itself (when its harness library is present) on the fixture inputs."""
    g = load("t4")
    ref = orc_mod.RefLib("t4")
    ref.set_links(g["u"])
    assert np.array_equal(ref.doe(g["x"]), g["doe"])
    ref.set_chi(np.stack([g["x"]] * ref.no_ps))
    assert np.array_equal(ref.msolve(1e-10, g["ms_shifts"])[0], g["ms_x"])
