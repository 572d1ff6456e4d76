"""The drop-in boundary exercised the way a reference user would: a C program written against the
reference's gate API (tests/c/dropin_gates.c) is compiled with gcc against include/tfhe.h, linked
with libtfhe_b200.so and run; every gate must decrypt to its truth table, in both precision forms and
for both of the reference's default parameter sets.  A second program (tests/c/dropin_threads.c) runs
gates from several threads at once on one keyset."""
import os
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("dropin") / "dropin_gates")
    libdir = os.path.join(ROOT, "tfhe_b200")
    subprocess.check_call(["gcc", "-std=c99", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "c", "dropin_gates.c"), "-o", exe, "-L", libdir,
                           "-ltfhe_b200", f"-Wl,-rpath,{libdir}"])
    return exe


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("lam", [110, 80])  # the 128-bit default and the 80-bit set
def test_c_program_against_dropin_header(program, precision, lam):
    res = subprocess.run([program, str(precision), str(lam)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.strip().endswith("OK")


@pytest.fixture(scope="module")
def threaded_program(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("dropin_threads") / "dropin_threads")
    libdir = os.path.join(ROOT, "tfhe_b200")
    subprocess.check_call(["gcc", "-std=c99", "-D_POSIX_C_SOURCE=200809L", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "c", "dropin_threads.c"), "-o", exe, "-L", libdir,
                           "-ltfhe_b200", f"-Wl,-rpath,{libdir}", "-lpthread"])
    return exe


@pytest.mark.parametrize("precision", [0, 1])
def test_concurrent_threads_on_one_keyset(threaded_program, precision):
    # four threads start together on a keyset whose key is not yet on the GPU
    res = subprocess.run([threaded_program, str(precision)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    assert res.stdout.strip().endswith("OK")
