"""The reference's own host program on this library: its unmodified lib/ sources compiled with
USE_GPU (update.cc:58-152 -> gpu.cc:10-31, cu_inverter.cc:21-72, fermionforce.cc, ipdot.cc,
momenta.cc, rationalapprox.cc) and linked against librhmc_b200.so in place of its lib/Cuda,
against the same sources compiled for the CPU.  Both draw their momenta, pseudofermions and
Metropolis uniforms from the reference's own RNG with the same seed, from the same cold start.

Bounds, per trajectory: identical accept/reject decisions; |Delta S_gpu - Delta S_cpu| <= 1e-4
and plaquettes within 1e-6.  The reference's GPU data contract moves momenta and ipdot between
host and device as single floats (packer.cc:443-566) and the force numerators as floats
(cuda_fermion_force.h:4), so the GPU trajectory starts from momenta rounded to 2^-24 relative:
over 4V x 8 momentum components that shifts the kinetic term by ~1e-6 and the MD evolution by
about as much.
"""
import os

import pytest

from dropin_util import binary, run

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag", ["t4", "a6448"])
def test_reference_update_on_librhmc(tag, tmp_path):
    if not (os.path.exists(binary(tag, False)) and os.path.exists(binary(tag, True))):
        pytest.skip("drop-in programs not built (oracle/dropin/build_dropin.py)")
    ntraj = 5
    cpu, _ = run(tag, False, ntraj, str(tmp_path))
    gpu, out = run(tag, True, ntraj, str(tmp_path))
    print("\n%s cpu %s\n%s gpu %s" % (tag, cpu, tag, gpu))
    assert [t[1] for t in gpu] == [t[1] for t in cpu]
    for (dc, _, pc, tc), (dg, _, pg, tg) in zip(cpu, gpu):
        assert abs(dg - dc) <= 1e-4, (dc, dg)
        assert abs(pg - pc) <= 1e-6 and abs(tg - tc) <= 1e-6, ((pc, tc), (pg, tg))
    if tag == "t4":  # this run exercises both outcomes of the Metropolis test
        assert {t[1] for t in cpu} == {0, 1}
