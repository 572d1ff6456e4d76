"""The LWE helpers of the reference's API (lwe-functions.h, approxPhase) and the batched torus
encrypt / decrypt of the native ABI.  Host side, no GPU, except the bootstrap checks marked gpu.
"""
import ctypes
import os
import subprocess

import numpy as np
import pytest

import tfhe_b200 as tb
from tfhe_ref import REF_DIR

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("lwe") / "dropin_lwe")
    libdir = os.path.join(ROOT, "tfhe_b200")
    subprocess.check_call(["gcc", "-std=c99", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "c", "dropin_lwe.c"), "-o", exe,
                           "-L", libdir, "-ltfhe_b200", "-Wl,-rpath," + libdir])
    return exe


def test_lwe_helpers_from_c(program):
    res = subprocess.run([program, "host"], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr


@pytest.mark.gpu
def test_coefficient_domain_bootstrap_from_c(program):
    res = subprocess.run([program, "gpu"], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr


def test_approx_phase_equals_the_reference():
    path = os.path.join(REF_DIR, "libtfhe-spqlios-fma.so")
    if not os.path.exists(path):
        pytest.skip("reference build (oracle/_ref) not present")
    ref = ctypes.CDLL(path)
    ours = tb.api.lib()
    for L in (ref, ours):
        L.approxPhase.restype = ctypes.c_int32
        L.approxPhase.argtypes = [ctypes.c_int32, ctypes.c_int32]
    rng = np.random.default_rng(4)
    for msize in (2, 3, 8, 17, 1024, 2**20):
        for ph in rng.integers(-2**31, 2**31, 200):
            assert ours.approxPhase(int(ph), msize) == ref.approxPhase(int(ph), msize)


def test_batched_torus_encrypt_decrypt():
    L = tb.api.lib()
    L.tfheb_encrypt_torus.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_double,
                                      ctypes.c_uint64, ctypes.c_void_p]
    L.tfheb_decrypt_torus.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int32, ctypes.c_int32,
                                      ctypes.c_void_p]
    p = tb.make_params(100, 1024, 1, 3, 7, 8, 2)
    sk, _ = tb.keygen(p, seed=3)
    msize = 16
    k = np.random.default_rng(2).integers(0, msize, 300)
    mu = ((k.astype(np.uint64) << 32) // msize).astype(np.uint32).view(np.int32)  # k / msize on the torus
    cts = np.zeros((len(k), p.n + 1), np.int32)
    assert L.tfheb_encrypt_torus(sk.h, mu.ctypes.data, len(k), 2.0**-15, 9, cts.ctypes.data) == 0
    out = np.zeros(len(k), np.int32)
    assert L.tfheb_decrypt_torus(sk.h, cts.ctypes.data, len(k), msize, out.ctypes.data) == 0
    assert (out == mu).all()
    # the phases carry the noise: small, not zero
    _, ph = sk.decrypt(cts)
    d = (ph.astype(np.int64) - mu.astype(np.int64) + 2**31) % 2**32 - 2**31
    assert 0 < np.abs(d).max() < 2**22
