"""Helpers for the drop-in tests: the reference's own host program built twice by
oracle/dropin/build_dropin.py (CPU code path, and GPU code path linked against librhmc_b200),
its coefficient file, and the parsing of its output."""
import json
import os
import re
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
REF = os.path.join(ROOT, "oracle", "_ref")


def binary(tag, gpu):
    return os.path.join(REF, "dropin_%s_%s" % ("gpu" if gpu else "cpu", tag))


def write_coeffs(tag, path):
    """The fixture approximations of configuration `tag` (normalised, as rationalapprox_calc would
    leave them) and the fixed eigenvalue bounds, in the format dropin_main.cc reads."""
    with open(os.path.join(HERE, "golden", "rational_coeffs.json")) as f:
        cf = json.load(f)[tag]
    g = np.load(os.path.join(HERE, "golden", "ref_%s.npz" % tag))
    with open(path, "w") as f:
        f.write("bounds %.17g %.17g\n" % tuple(float(v) for v in g["bounds"]))
        for w, c in enumerate(cf):
            f.write("approx %d %d %.17g %.17g\n" % (w, len(c["a"]), c["min_eps"], c["a0"]))
            f.write(" ".join("%.17g" % v for v in c["a"]) + "\n")
            f.write(" ".join("%.17g" % v for v in c["b"]) + "\n")


def run(tag, gpu, ntraj, workdir, timeout=600):
    """Runs the program in workdir (it writes its data and error files there); returns a list of
    (delta_s, accepted, plaq_spatial, plaq_temporal) per trajectory and the raw output."""
    coeffs = os.path.join(workdir, "coeffs_%s.txt" % tag)
    write_coeffs(tag, coeffs)
    env = dict(os.environ, RHMC_DROPIN_COEFFS=coeffs)
    r = subprocess.run([binary(tag, gpu), str(ntraj)], cwd=workdir, env=env, capture_output=True, text=True,
                       timeout=timeout)
    assert r.returncode == 0, (r.returncode, r.stdout[-2000:], r.stderr[-2000:])
    ds = [float(m) for m in re.findall(r"Delta S = (\S+)", r.stdout)]
    traj = re.findall(r"TRAJ (\d+) acc (-?\d+) plaq (\S+) (\S+)", r.stdout)
    assert len(ds) == ntraj and len(traj) == ntraj, r.stdout[-2000:]
    return [(ds[i], int(traj[i][1]), float(traj[i][2]), float(traj[i][3])) for i in range(ntraj)], r.stdout
