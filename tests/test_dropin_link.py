"""The reference's own host sources, compiled with USE_GPU by oracle/dropin/build_dropin.py, link
against librhmc_b200.so with every symbol resolved: the entry points its gpu.cc, cu_inverter.cc,
fermionforce.cc, ipdot.cc, momenta.cc and rationalapprox.cc call (lib/Cuda/*.h) are exported by
the library under the same names (no GPU needed: the loader only resolves symbols)."""
import os
import subprocess

import pytest

from dropin_util import ROOT, binary

LIB = os.path.join(ROOT, "rhmc-on-gpu_b200", "librhmc_b200.so")


def _undefined(path):
    out = subprocess.run(["nm", "-D", "--undefined-only", path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1].split("@")[0] for line in out.splitlines() if line.strip()}


def _exported(path):
    out = subprocess.run(["nm", "-D", "--defined-only", path], capture_output=True, text=True, check=True).stdout
    return {line.split()[-1].split("@")[0] for line in out.splitlines() if line.strip()}


@pytest.mark.parametrize("tag", ["t4", "a6448"])
def test_reference_gpu_host_code_links(tag):
    b = binary(tag, True)
    if not os.path.exists(b):
        pytest.skip("drop-in programs not built (oracle/dropin/build_dropin.py)")
    need = {s for s in _undefined(b) if s.startswith("cuda_") or s.startswith("rhmc_")}
    # the reference's GPU glue calls at least the solver, force, update and transfer entry points
    assert {"cuda_init0", "cuda_init1", "cuda_end", "cuda_shifted_inverter", "cuda_shifted_inverter_d",
            "cuda_sol_sum", "cuda_fermion_force", "cuda_gauge_deriv", "cuda_exp_su3",
            "cuda_momenta_sum_multiply"} <= need
    assert need <= _exported(LIB), need - _exported(LIB)
    r = subprocess.run(["ldd", "-r", b], capture_output=True, text=True)
    assert "undefined symbol" not in r.stdout + r.stderr, r.stdout + r.stderr
