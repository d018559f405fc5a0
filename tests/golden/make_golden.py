#!/usr/bin/env python3
"""Generate the golden fixtures from the reference's own CPU code.

Runs the unmodified reference sources (compiled by oracle/build_ref.py into
oracle/_ref/libref_<tag>.so) on seeded synthetic inputs and records inputs and outputs in
tests/golden/ref_<tag>.npz, plus the rational coefficients both sides use in
tests/golden/rational_coeffs.json.  Needs the reference checkout only to build the harness;
the fixtures it writes are what the tests read (the GPU box has no reference checkout).

Usage: python tests/golden/make_golden.py [--build]
"""
import argparse
import json
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "rhmc-on-gpu_b200"))

from rhmc_b200 import fields as F  # noqa: E402
from rhmc_b200 import rational as R  # noqa: E402

# spectral bounds handed to findminmax's replacement, per build (mass^2 <= lambda <= 16 + mass^2)
BOUNDS = {"t4": (0.01, 16.0), "a6448": (0.04, 16.0)}
# (first power, first degree), (md power, md degree), (last power, last degree) per build
APPROX = {"t4": ((0.25, 8), (-0.5, 8), (-0.5, 8)), "a6448": ((0.125, 8), (-0.25, 6), (-0.25, 8))}
EPS = 1e-4
UNIFORM = 0.5


def coefficients():
    path = os.path.join(HERE, "rational_coeffs.json")
    if os.path.exists(path):
        with open(path) as f:
            return json.load(f)
    out = {}
    for tag, specs in APPROX.items():
        out[tag] = [R.rational_power(p, n, EPS) for p, n in specs]
    with open(path, "w") as f:
        json.dump(out, f, indent=1)
    return out


def make(tag, coeffs):
    import oracle
    ref = oracle.RefLib(tag)
    dims = ref.dims
    out = {"dims": np.array(dims), "mass": ref.mass, "beta": ref.beta, "no_ps": ref.no_ps, "no_md": ref.no_md,
           "gauge_scale": ref.gauge_scale, "no_flavours": ref.no_flavours, "bounds": np.array(BOUNDS[tag]),
           "uniform": UNIFORM, "residue_md": ref.residue_md, "residue_metro": ref.residue_metro}
    u = F.random_links(dims, seed=1001)
    P = F.random_momenta(dims, seed=3003)
    phi = F.random_spinor(dims, seed=2002, n=ref.no_ps)
    x = F.random_spinor(dims, seed=4004)
    out.update(u=u, P=P, phi=phi, x=x)
    t, e = ref.tables()
    out.update(table=t, eta=e)
    ref.set_links(u)
    out["doe"] = ref.doe(x)
    out["deo"] = ref.deo(x)
    shifts = np.geomspace(2e-3, 30.0, 5)
    chi = np.stack([x] * ref.no_ps)
    ref.set_chi(chi)
    out["ms_shifts"] = shifts
    out["ms_x"] = ref.msolve(1e-10, shifts)[0]
    for w, c in enumerate(coeffs[tag]):
        ref.set_approx(w, c)
    ref.set_minmax(*BOUNDS[tag])
    # heatbath, forces, updates
    ref.set_phi(phi)
    ref.lib.ref_first_inv_approx_calc(1e-10)
    out["chi"] = ref.get_chi()
    ref.set_links(u)
    ref.lib.ref_calc_ipdot_gauge()
    out["ipdot_gauge"] = ref.get_ipdot()
    ref.lib.ref_calc_ipdot_fermion()
    out["ipdot_fermion"] = ref.get_ipdot()
    ref.lib.ref_calc_ipdot()
    out["ipdot_full"] = ref.get_ipdot()
    ref.set_momenta(P)
    ref.lib.ref_mom_update(-0.05)
    out["P_after"] = ref.get_momenta()
    ref.lib.ref_link_update(0.05)
    out["u_after"] = ref.get_links()
    ref.set_links(u)
    s, tp = ref.plaquette()
    out["plaq"] = np.array([s, tp])
    # one trajectory per integrator from the same start
    for integ in range(4):
        ref.set_links(u)
        ref.set_momenta(P)
        ref.set_phi(phi)
        de, acc = ref.trajectory(integ, UNIFORM)
        out["traj%d_de" % integ] = de
        out["traj%d_acc" % integ] = acc
        out["traj%d_plaq" % integ] = np.array(ref.plaquette())
        if integ == 0:
            out["traj0_u"] = ref.get_links()
    np.savez_compressed(os.path.join(HERE, "ref_%s.npz" % tag), **out)
    print(tag, "written", {k: (v.shape if hasattr(v, "shape") else v) for k, v in out.items() if k.startswith("traj")})


def make_packer(tag):
    """The reference packer (lib/Tools/Packer/packer.cc, compiled unmodified into the harness as
    refpk_*) on the fixture fields of ref_<tag>.npz: every packed host format the GPU entry
    points exchange, and the reference's unpacking of packed buffers."""
    import oracle
    g = dict(np.load(os.path.join(HERE, "ref_%s.npz" % tag)))
    ref = oracle.RefLib(tag)
    out = {}
    ref.set_links(g["u"])
    out["pk_gauge"] = ref.pk_gauge()
    ref.set_chi(g["chi"])
    out["pk_chi"] = ref.pk_chi()
    out["pk_fermion"] = ref.pk_fermion(g["x"])
    out["pk_fermion_d"] = ref.pk_fermion_d(g["x"])
    ref.set_ipdot(g["ipdot_full"])
    out["pk_tamatrix"] = ref.pk_ipdot()
    ref.set_momenta(g["P"])
    out["pk_thmatrix"] = ref.pk_momenta()
    out["shift_table"] = ref.shift_table()
    # unpacking: of the packed buffers above (the gauge one with its unitarize_with_eta)
    out["unpk_gauge"] = ref.unpk_gauge(out["pk_gauge"])
    out["unpk_chi"] = ref.unpk_chi(out["pk_chi"])
    out["unpk_fermion_d"] = ref.unpk_fermion_d(out["pk_fermion_d"])
    out["unpk_tamatrix"] = ref.unpk_ipdot(out["pk_tamatrix"])
    out["unpk_thmatrix"] = ref.unpk_momenta(out["pk_thmatrix"])
    np.savez_compressed(os.path.join(HERE, "ref_%s_packer.npz" % tag), **out)
    print(tag, "packer fixture written", sorted(out))


def make_meas(tag, ncalls=2):
    """The reference's measurements on the fixture links of ref_<tag>.npz: Conf::calc_poly and
    ncalls calls of chiral_meas (rand_vect = 1), each with the Z2 noise it drew (copied out of the
    reference after the call) and its chiral condensate, energy, baryon and pressure densities."""
    import oracle
    g = dict(np.load(os.path.join(HERE, "ref_%s.npz" % tag)))
    ref = oracle.RefLib(tag)
    ref.set_links(g["u"])
    out = {"polyakov": np.array(ref.polyakov())}
    res, ne, no = [], [], []
    for _ in range(ncalls):
        r, e, o = ref.chiral_meas()
        res.append(r)
        ne.append(e)
        no.append(o)
    out["chiral"] = np.array(res)
    out["noise_e"] = np.array(ne)
    out["noise_o"] = np.array(no)
    # the configuration file the reference writes for these links, and what its reader makes of
    # it (4^4 only, to keep the fixtures small)
    if tag == "t4":
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            out["conf_text"] = np.frombuffer(ref.write_conf(d), np.uint8)
            out["conf_read"] = ref.read_conf(d)
    out["residue_metro"] = np.array(ref.param(3))
    out["no_flavours"] = np.array(ref.param(2))
    np.savez_compressed(os.path.join(HERE, "ref_%s_meas.npz" % tag), **out)
    print(tag, "measurement fixture written", sorted(out))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--build", action="store_true", help="(re)build the reference harness first")
    ap.add_argument("--packer-only", action="store_true", help="only the packed-format fixture")
    ap.add_argument("--meas-only", action="store_true", help="only the measurement fixtures")
    a = ap.parse_args()
    if a.build:
        subprocess.check_call([sys.executable, os.path.join(ROOT, "oracle", "build_ref.py"), "t4", "a6448"])
    if a.meas_only:
        for tag in ("t4", "a6448"):
            make_meas(tag)
        return
    if not a.packer_only:
        coeffs = coefficients()
        for tag in ("t4", "a6448"):
            make(tag, coeffs)
    make_packer("t4")
    for tag in ("t4", "a6448"):
        make_meas(tag)


if __name__ == "__main__":
    main()
