"""Measurements on the device (rhmc_polyakov, rhmc_chiral_meas) against the reference's own
outputs (tests/golden/ref_<tag>_meas.npz, with the Z2 noise the reference drew).  The Polyakov
loop multiplies the same links in the same order as Conf::calc_poly (tolerance 1e-13); the
chiral measurement solves to the absolute residual 1e-10 like the reference's CG (different start
vectors), so its results agree to 1e-9 absolute on values of order 1."""
import os

import numpy as np
import pytest

import rhmc_b200 as rb

pytestmark = pytest.mark.gpu
HERE = os.path.dirname(os.path.abspath(__file__))
TAGS = ["t4", "a6448"]


def _setup(tag):
    from gpu_util import new_ctx
    g = dict(np.load(os.path.join(HERE, "golden", "ref_%s.npz" % tag)))
    m = dict(np.load(os.path.join(HERE, "golden", "ref_%s_meas.npz" % tag)))
    ctx = new_ctx(tuple(int(d) for d in g["dims"]), mass=float(g["mass"]), beta=float(g["beta"]))
    ctx.set_gauge(g["u"])
    return g, m, ctx


@pytest.mark.parametrize("tag", TAGS)
def test_polyakov(tag):
    g, m, ctx = _setup(tag)
    re, im = ctx.polyakov()
    assert abs(re - m["polyakov"][0]) < 1e-13 and abs(im - m["polyakov"][1]) < 1e-13


@pytest.mark.parametrize("tag", TAGS)
def test_chiral_meas(tag):
    g, m, ctx = _setup(tag)
    nf, res = int(m["no_flavours"]), float(m["residue_metro"])
    for call in range(m["chiral"].shape[0]):
        got = ctx.chiral_meas(m["noise_e"][call], m["noise_o"][call], residual=res, no_flavours=nf)
        assert np.max(np.abs(got - m["chiral"][call])) < 1e-9, (call, got, m["chiral"][call])
    # several noise pairs in one call: the average of the single-pair results
    both = ctx.chiral_meas(m["noise_e"], m["noise_o"], residual=res, no_flavours=nf)
    assert np.max(np.abs(both - m["chiral"].mean(axis=0))) < 1e-9


def test_chiral_meas_errors():
    g, m, ctx = _setup("t4")
    with pytest.raises(rb.RhmcError):
        ctx.chiral_meas(m["noise_e"][0], m["noise_o"][0], residual=0.0)


def test_conf_write_matches_reference_text(tmp_path):
    # the same links written by the library and by Conf::write_last: identical text
    g, m, ctx = _setup("t4")
    path = tmp_path / "conf"
    ctx.write_conf(path, no_flavours=2, update_iteration=0)
    assert path.read_bytes() == bytes(m["conf_text"])


def test_conf_read(tmp_path):
    import sys
    sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
    import oracle
    g, m, ctx = _setup("t4")
    path = tmp_path / "config"
    path.write_bytes(bytes(m["conf_text"]))
    # as the reference reads it (no reunitarisation): the stored numbers exactly
    hdr = ctx.read_conf(path, reunitarize=0)
    assert hdr == {"beta": 5.5, "mass": 0.1, "no_flavours": 2, "update_iteration": 0}
    assert np.array_equal(ctx.get_gauge(), m["conf_read"])
    # with the reunitarisation the reference's reader means to apply (Conf::unitarize_with_eta)
    ctx.read_conf(path, reunitarize=1)
    orc = oracle.Oracle(tuple(int(d) for d in g["dims"]))
    want = orc.unitarize_with_eta(m["conf_read"].copy())
    assert np.max(np.abs(ctx.get_gauge() - want)) < 1e-15


def test_conf_read_errors(tmp_path):
    from gpu_util import new_ctx
    _, m, ctx = _setup("t4")
    path = tmp_path / "config"
    path.write_bytes(bytes(m["conf_text"]))
    other = new_ctx((4, 4, 4, 6))
    with pytest.raises(rb.RhmcError):
        other.read_conf(path)  # stored_conf_not_fit
    bad = tmp_path / "short"
    bad.write_bytes(bytes(m["conf_text"])[:5000])
    with pytest.raises(rb.RhmcError):
        ctx.read_conf(bad)  # truncated link data
    with pytest.raises(rb.RhmcError):
        ctx.read_conf(tmp_path / "missing")
