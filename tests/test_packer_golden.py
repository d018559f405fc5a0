"""The packed host formats of the legacy GPU boundary (lib/Tools/Packer/packer.cc) against the
reference packer itself: tests/golden/ref_t4_packer.npz was recorded by running the unmodified
packer.cc on the 4^4 fixture fields (tests/golden/make_golden.py).  tests/legacy_pack.py -- the
restatement the legacy GPU tests build their buffers with -- must reproduce every packed buffer
and every unpacked field bit for bit.  CPU only."""
import os

import numpy as np
import pytest

import legacy_pack as LP
from rhmc_b200 import fields as F

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def fx():
    g = dict(np.load(os.path.join(HERE, "golden", "ref_t4.npz")))
    pk = dict(np.load(os.path.join(HERE, "golden", "ref_t4_packer.npz")))
    return g, pk


def same_bits(a, b):
    a, b = np.ascontiguousarray(a), np.ascontiguousarray(b)
    return a.dtype == b.dtype and a.shape == b.shape and np.array_equal(a.view(np.uint8), b.view(np.uint8))


def test_pack_formats(fx):
    g, pk = fx
    assert same_bits(LP.pack_gauge(g["u"]), pk["pk_gauge"])
    assert same_bits(LP.pack_multifermion(g["chi"]), pk["pk_chi"])
    assert same_bits(LP.pack_fermion(g["x"]), pk["pk_fermion"])
    assert same_bits(LP.pack_fermion_d(g["x"]), pk["pk_fermion_d"])
    assert same_bits(LP.pack_tamatrix(g["ipdot_full"]), pk["pk_tamatrix"])
    assert same_bits(LP.pack_thmatrix(g["P"]), pk["pk_thmatrix"])


def test_unpack_formats(fx):
    import oracle
    g, pk = fx
    V = int(np.prod(g["dims"]))
    # smartunpack_gauge = rows 0-1 from hi + lo, then Conf::unitarize_with_eta (conf.cc:235-251)
    u = np.zeros((4 * V, 3, 3), np.complex128)
    u[:, :2, :] = LP.unpack_gauge_rows01(pk["pk_gauge"], V)
    oracle.Oracle(tuple(g["dims"])).unitarize_with_eta(u)
    assert same_bits(u, pk["unpk_gauge"])
    assert same_bits(LP.unpack_multifermion(pk["pk_chi"], 1, V // 2), pk["unpk_chi"])
    assert same_bits(LP.unpack_multifermion(pk["pk_fermion_d"], 1, V // 2)[0], pk["unpk_fermion_d"])
    assert same_bits(LP.unpack_alg(pk["pk_tamatrix"], V, True), pk["unpk_tamatrix"])
    assert same_bits(LP.unpack_alg(pk["pk_thmatrix"], V, False), pk["unpk_thmatrix"])


def test_shift_table(fx):
    """make_shift_table (packer.cc:415-439) against the table the library's geometry and the
    legacy tests use."""
    g, pk = fx
    assert np.array_equal(F.neighbour_table(tuple(g["dims"])), pk["shift_table"])


@pytest.mark.skipif(not os.path.exists(os.path.join(os.path.dirname(HERE), "oracle", "_ref", "libref_t4.so")),
                    reason="reference harness not built")
def test_reference_packer_live(fx):
    """Re-run the reference packer (when the harness library is present) on fresh random fields."""
    import oracle
    g, _ = fx
    dims = tuple(g["dims"])
    ref = oracle.RefLib("t4")
    u = F.random_links(dims, seed=99)
    ref.set_links(u)
    assert same_bits(ref.pk_gauge(), LP.pack_gauge(u))
    x = F.random_spinor(dims, seed=98)
    assert same_bits(ref.pk_fermion_d(x), LP.pack_fermion_d(x))
    P = F.random_momenta(dims, seed=97)
    ref.set_momenta(P)
    assert same_bits(ref.pk_momenta(), LP.pack_thmatrix(P))
