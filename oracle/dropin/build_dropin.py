#!/usr/bin/env python3
"""Build the reference's own host program against librhmc_b200 -- TEST INFRASTRUCTURE ONLY.

Compiles the unmodified sources of coppolachan/RHMC-on-GPU (its lib/ tree, as it lies in the
reference checkout) with oracle/dropin/dropin_main.cc as the main program, twice per lattice
configuration of oracle/build_ref.py:

  oracle/_ref/dropin_cpu_<tag>   without USE_GPU: the reference's CPU code path;
  oracle/_ref/dropin_gpu_<tag>   with -DUSE_GPU, linked against rhmc-on-gpu_b200/librhmc_b200.so
                                 in place of the reference's lib/Cuda directory (which is not
                                 compiled): the reference's GPU code path on this library.

Left out of both: lib/Main/rhmc.cc (dropin_main.cc is the main program), the Remez generator
(alg_remez.cc, rationalapprox_calc.cc, test_rational_approx.cc: MPFR/GMP headers are absent;
dropin_main.cc reads the coefficients instead), findminmax.cc (fixed bounds in dropin_main.cc,
so both builds rescale identically) and revupdate.cc (compiled only for REVERSIBILITY_TEST).
Everything else, including lib/Main/init.cc, lib/Main/Gpu/gpu.cc,
lib/Action/Inverter/cu_inverter.cc and the packer, is compiled unmodified.

The reference sources are found as oracle/build_ref.py finds them (--ref, RHMC_REFERENCE_SRC,
or that script's default); without them nothing is built.  Outputs go only to oracle/_ref/.
Usage: python oracle/dropin/build_dropin.py [--ref DIR] [tag ...]     (default tags: t4 a6448)
"""
import argparse
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE = os.path.dirname(HERE)
ROOT = os.path.dirname(ORACLE)
sys.path.insert(0, ORACLE)
import build_ref as BR  # noqa: E402

OUT = BR.OUT
PKG = os.path.join(ROOT, "rhmc-on-gpu_b200")
EXCLUDE = {
    "lib/Main/rhmc.cc", "lib/Tools/RationalApprox/alg_remez.cc", "lib/Tools/RationalApprox/rationalapprox_calc.cc",
    "lib/Tools/RationalApprox/test_rational_approx.cc", "lib/Action/Findminmax/findminmax.cc",
    "lib/Update/RevUpdate/revupdate.cc",
}


def sources(ref):
    out = []
    for root, _, files in os.walk(os.path.join(ref, "lib")):
        for f in files:
            if f.endswith(".cc") or f.endswith(".c"):
                rel = os.path.relpath(os.path.join(root, f), ref)
                if rel not in EXCLUDE:
                    out.append(rel)
    return sorted(out)


def binary(tag, gpu):
    return os.path.join(OUT, "dropin_%s_%s" % ("gpu" if gpu else "cpu", tag))


def up_to_date(tag, gpu):
    b = binary(tag, gpu)
    if not os.path.exists(b):
        return False
    deps = [os.path.abspath(__file__), os.path.join(HERE, "dropin_main.cc"), os.path.join(ORACLE, "build_ref.py")]
    if gpu:
        deps.append(os.path.join(PKG, "librhmc_b200.so"))
    return all(os.path.getmtime(b) >= os.path.getmtime(d) for d in deps if os.path.exists(d))


def build(ref, tag, gpu, jobs=8):
    cfg = BR.CONFIGS[tag]
    bdir = os.path.join(OUT, "build_dropin_%s_%s" % ("gpu" if gpu else "cpu", tag))
    os.makedirs(os.path.join(bdir, "include"), exist_ok=True)
    with open(os.path.join(bdir, "include", "parameters.h"), "w") as f:
        f.write(BR.PARAM_TEMPLATE.format(tag=tag, **cfg))
    defs = ["-DUSE_GPU"] if gpu else []
    inc = ["-I" + bdir, "-I" + ref, "-I" + os.path.join(ROOT, "include")]
    objs, cmds = [], []
    for rel in sources(ref) + ["MAIN"]:
        src = os.path.join(HERE, "dropin_main.cc") if rel == "MAIN" else os.path.join(ref, rel)
        obj = os.path.join(bdir, rel.replace("/", "_") + ".o")
        objs.append(obj)
        if src.endswith(".c"):
            cmds.append(["gcc", "-O2", "-fPIC", "-ffp-contract=off", "-w"] + defs + inc + ["-c", src, "-o", obj])
        else:
            cmds.append(["g++"] + BR.CXXFLAGS + defs + inc + ["-c", src, "-o", obj])

    def run(c):
        r = subprocess.run(c, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("failed: %s\n%s" % (" ".join(c), r.stderr[-4000:]))

    with ThreadPoolExecutor(jobs) as ex:
        list(ex.map(run, cmds))
    link = ["g++", "-o", binary(tag, gpu)] + objs
    if gpu:
        # the library is found next to the checkout at run time, wherever the checkout lies
        link += ["-L" + PKG, "-lrhmc_b200", "-Wl,-rpath,$ORIGIN/../../rhmc-on-gpu_b200"]
    run(link)
    shutil.rmtree(bdir, ignore_errors=True)
    return binary(tag, gpu)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("RHMC_REFERENCE_SRC", BR.DEFAULT_REF))
    ap.add_argument("--force", action="store_true")
    ap.add_argument("tags", nargs="*")
    a = ap.parse_args()
    if not os.path.isdir(os.path.join(a.ref, "lib")):
        print("reference sources not found at %s; nothing built" % a.ref)
        return 0
    if not os.path.exists(os.path.join(PKG, "librhmc_b200.so")):
        print("librhmc_b200.so not built; run make -C rhmc-on-gpu_b200 first")
        return 1
    os.makedirs(OUT, exist_ok=True)
    for tag in (a.tags or ["t4", "a6448"]):
        for gpu in (False, True):
            if not a.force and up_to_date(tag, gpu):
                print("up to date", binary(tag, gpu))
                continue
            print("built", build(a.ref, tag, gpu))
    return 0


if __name__ == "__main__":
    sys.exit(main())
