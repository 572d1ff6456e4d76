"""The reference's scalar blind-rotation, external-product and keyswitch API through the drop-in
header, checked against the reference library built from its sources (oracle/_ref).

tests/c/dropin_rotate.c, compiled against include/tfhe.h, loads a secret keyset that the reference
wrote (tfhe_io.cpp format) and checks the entry points against each other bit for bit
(tfhe_blindRotate(_FFT), tfhe_blindRotateAndExtract_FFT, tGswExternProduct, tGswExternMulToTLwe,
tfhe_bootstrap(_FFT), lweKeySwitch).  It records inputs and outputs; here the reference recomputes:
  * lweKeySwitch (lwe-keyswitch-functions.cpp:228-238) of the extracted samples: the drop-in's
    tfhe_bootstrap_FFT and bootsNAND outputs must equal it bit for bit, and their current_variance
    must equal the reference's (the keyswitching-key variances summed over the non-zero digits);
  * tGswExternProduct (tgsw-functions.cpp:416-431) on the same key sample and input: equal within the
    precision form's product error (the reference's FFT products truncate), and the same
    current_variance (digit norms times row variances, plus the input's).
"""
import os
import subprocess

import numpy as np
import pytest

from tfhe_oracle import torus_diff
from tfhe_ref import RefLib

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not RefLib.available(), reason="reference build (oracle/_ref) not present")]
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def program(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("dropin_rotate") / "dropin_rotate")
    libdir = os.path.join(ROOT, "tfhe_b200")
    subprocess.check_call(["gcc", "-std=c99", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "c", "dropin_rotate.c"), "-o", exe, "-L", libdir,
                           "-ltfhe_b200", f"-Wl,-rpath,{libdir}"])
    return exe


@pytest.fixture(scope="module")
def ref_keys(tmp_path_factory):
    keys = RefLib.load().keygen(custom=None, seed=2718)
    path = str(tmp_path_factory.mktemp("keys") / "secret.key")
    keys.save_secret_keyset(path)
    yield keys, path
    keys.free()


class Reader:
    def __init__(self, path):
        self.buf = open(path, "rb").read()
        self.pos = 0

    def i32(self, count):
        out = np.frombuffer(self.buf, np.int32, count, self.pos).copy()
        self.pos += 4 * count
        return out

    def f64(self):
        out = float(np.frombuffer(self.buf, np.float64, 1, self.pos)[0])
        self.pos += 8
        return out

    def done(self):
        return self.pos == len(self.buf)


@pytest.mark.parametrize("precision", [0, 1])
def test_scalar_rotation_api_against_reference(program, ref_keys, tmp_path, precision, oracle):
    keys, key_path = ref_keys
    _, _, _, bsk = keys.export(ksk=False)
    rec_path = str(tmp_path / "record.bin")
    res = subprocess.run([program, key_path, rec_path, str(precision)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    n, N, k = keys.n, keys.N, keys.k
    kN, tl = k * N, (k + 1) * N
    r = Reader(rec_path)
    trials = 0
    while not r.done():
        x0, x1 = r.i32(n + 1), r.i32(n + 1)
        u0 = r.i32(kN + 1)
        y0, y0_var = r.i32(n + 1), r.f64()
        y1, y1_var = r.i32(n + 1), r.f64()
        u2 = r.i32(kN + 1)
        g, g_var = r.i32(n + 1), r.f64()
        step = int(r.i32(1)[0])
        b, b_var = r.i32(tl), r.f64()
        prod, prod_var = r.i32(tl), r.f64()
        trials += 1

        # keyswitch of the extracted samples, and its variance bookkeeping
        want, want_var = keys.keyswitch(np.stack([u0, u2]), with_variance=True)
        assert (y0 == want[0]).all(), "tfhe_bootstrap_FFT differs from the reference's lweKeySwitch of its sample"
        assert (y1 == want[0]).all()
        assert y0_var == want_var[0] and y1_var == want_var[0], (y0_var, y1_var, want_var[0])
        assert (g == want[1]).all(), "bootsNAND differs from the reference's lweKeySwitch of its sample"
        assert g_var == want_var[1]
        bits, _ = keys.decrypt(np.stack([x0, x1, g]))
        assert bits[2] == 1 - (bits[0] & bits[1])

        # the external product on the same key sample.  The reference adds (k+1)l digit-row products,
        # each through its own FFT product rounded to Torus32 (tlwe-functions.cpp:191-197,
        # torusPolynomialAddMulRFFT), so it may be off the exact product by up to one unit per row;
        # this library rounds the sum once (FP64: within one unit of exact).  Against the exact
        # oracle: one unit (FP64) or the split form's stated bound; against the reference: those
        # plus one unit per row.
        ref_prod, ref_var = keys.extern_product(step, b, b_var)
        rows = (k + 1) * keys.l
        want_exact = oracle.external_product(keys.params(), bsk[step], b)
        e = np.abs(torus_diff(prod, want_exact))
        assert e.max() <= (1 if precision == 0 else 2**17), f"external product off the exact one by {e.max()} units"
        d = np.abs(torus_diff(prod, ref_prod))
        assert d.max() <= (rows + 1 if precision == 0 else 2**17), f"external product differs by {d.max()} units"
        assert prod_var == ref_var, (prod_var, ref_var)
    assert trials == 3
