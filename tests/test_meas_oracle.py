"""The oracle's restatement of the reference measurements (Polyakov loop, chiral condensate and
the energy, baryon and pressure densities) against the reference's own outputs recorded in
tests/golden/ref_<tag>_meas.npz (tests/golden/make_golden.py: the unmodified reference with its
own Z2 noise, which it records).  The reference solves with its CPU CG from a random start, the
oracle from zero, both to the absolute residual 1e-10, so the fermionic results agree to that
solver accuracy (tolerance 1e-9 absolute on values of order 1)."""
import os
import sys

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(os.path.dirname(HERE), "oracle"))
import oracle  # noqa: E402

TAGS = ["t4", "a6448"]


def _load(tag):
    g = dict(np.load(os.path.join(HERE, "golden", "ref_%s.npz" % tag)))
    m = dict(np.load(os.path.join(HERE, "golden", "ref_%s_meas.npz" % tag)))
    return g, m


@pytest.mark.parametrize("tag", TAGS)
def test_polyakov_matches_reference(tag):
    g, m = _load(tag)
    orc = oracle.Oracle(tuple(int(d) for d in g["dims"]))
    re, im = orc.polyakov(g["u"])
    assert abs(re - m["polyakov"][0]) < 1e-14 and abs(im - m["polyakov"][1]) < 1e-14


@pytest.mark.parametrize("tag", TAGS)
def test_chiral_meas_matches_reference(tag):
    g, m = _load(tag)
    orc = oracle.Oracle(tuple(int(d) for d in g["dims"]))
    for call in range(m["chiral"].shape[0]):
        got = orc.chiral_meas(g["u"], m["noise_e"][call], m["noise_o"][call], float(g["mass"]), int(m["no_flavours"]),
                              float(m["residue_metro"]))
        assert np.max(np.abs(got - m["chiral"][call])) < 1e-9, (call, got, m["chiral"][call])


def test_noise_is_z2():
    # the reference's noise: every colour component +-1 (Vec3::z2noise)
    _, m = _load("t4")
    for f in (m["noise_e"], m["noise_o"]):
        assert np.all(np.abs(f.real) == 1.0) and np.all(f.imag == 0.0)


def test_conf_fixture_self_consistent():
    # the reference's reader returns the numbers of its writer's text, parsed (correct rounding)
    _, m = _load("t4")
    text = bytes(m["conf_text"]).decode()
    tok = text.split()
    assert [int(t) for t in tok[:4]] == [4, 4, 4, 4] and tok[6] == "2" and tok[7] == "0"
    vals = np.array([complex(*map(float, t.strip("()").split(","))) for t in tok[8:]])
    assert np.array_equal(vals, m["conf_read"].reshape(-1))
