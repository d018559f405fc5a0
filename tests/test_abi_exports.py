"""The C ABI shared library loads on a host without a GPU and exports every function that
include/*.h declares (no compute calls: this runs on CPU)."""
import ctypes
import glob
import os
import re

import pytest

import rhmc_b200 as rb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_functions():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        text = open(h).read()
        text = re.sub(r"/\*.*?\*/", " ", text, flags=re.S)  # drop comments
        text = re.sub(r"typedef\s+struct\s*\{.*?\}\s*\w+\s*;", " ", text, flags=re.S)
        for m in re.finditer(r"\b(?:int|void|const\s+char\s*\*|rhmc_ctx\s*\*)\s*\**\s*(\w+)\s*\(", text):
            names.add(m.group(1))
    return sorted(names)


def test_headers_declare_the_boundary():
    names = declared_functions()
    for must in ("rhmc_create", "rhmc_dslash", "rhmc_msolve", "rhmc_fermion_force", "rhmc_gauge_force",
                 "rhmc_link_update", "rhmc_mom_update", "rhmc_update", "cuda_init0", "cuda_shifted_inverter_d",
                 "cuda_sol_sum", "cuda_fermion_force", "cuda_gauge_deriv", "cuda_exp_su3",
                 "cuda_momenta_sum_multiply", "cuda_find_max", "rhmc_true_residuals_noalloc"):
        assert must in names, must
    assert len(names) > 50


@pytest.mark.parametrize("name", declared_functions())
def test_library_exports(name):
    lib = rb.lib()  # ctypes.CDLL of the in-tree librhmc_b200.so
    assert isinstance(getattr(lib, name), ctypes._CFuncPtr)


def test_errors_without_a_context():
    lib = rb.lib()
    assert lib.rhmc_create(None, None) == -1  # RHMC_ERR_ARG
    assert b"null" in lib.rhmc_last_error()
    assert lib.rhmc_destroy(None) == 0


def test_headers_are_plain_c(tmp_path):
    """Both headers compile as pedantic C99 and a C program links against the library (the
    boundary needs no C++); destroying a null context is a no-op that returns RHMC_OK."""
    import shutil
    import subprocess
    if shutil.which("gcc") is None:
        pytest.skip("no C compiler")
    src = tmp_path / "abi.c"
    src.write_text('#include "rhmc_b200.h"\n#include "rhmc_legacy.h"\n'
                   "int main(void) { rhmc_params p = {4, 4, 4, 4, 0, 0.1, 5.5, 0}; (void)p;\n"
                   "  return rhmc_destroy((rhmc_ctx *)0); }\n")
    libdir = os.path.join(ROOT, "rhmc-on-gpu_b200")  # the in-tree build
    exe = tmp_path / "abi"
    subprocess.check_call(["gcc", "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-I" + os.path.join(ROOT, "include"),
                           str(src), "-L" + libdir, "-lrhmc_b200", "-Wl,-rpath," + libdir, "-o", str(exe)])
    assert subprocess.run([str(exe)]).returncode == 0
