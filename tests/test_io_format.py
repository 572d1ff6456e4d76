"""Files in the reference's format (tfhe_io.cpp): parameter sets, secret and cloud key sets and
ciphertexts move between the reference library and this one.  Host-only (no GPU).

The reference side is its own FILE* export/import functions, run from the reference build in
oracle/_ref; those tests skip when that build is absent.  Bars: what the reference writes loads
here bit-exact and is written back byte for byte; what this library writes loads in the
reference, which then decrypts and evaluates gates with it.
"""
import os
import subprocess

import numpy as np
import pytest

import tfhe_b200 as tb
from tfhe_b200.api import TfhebError
from tfhe_ref import RefLib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SMALL = dict(n=100, N=1024, k=1, l=3, Bgbit=7, ks_t=8, ks_basebit=2)


@pytest.fixture(scope="module")
def ref():
    r = RefLib.load()
    if r is None:
        pytest.skip("reference build (oracle/_ref) not present")
    return r


@pytest.fixture(scope="module")
def ref_keys(ref):
    k = ref.keygen(custom=SMALL, seed=77)
    yield k
    k.free()


def read(path):
    with open(path, "rb") as f:
        return f.read()


def small_params():
    return tb.make_params(*(SMALL[f] for f in ("n", "N", "k", "l", "Bgbit", "ks_t", "ks_basebit")))


# ---------------------------------------------------------------------------------------------
# parameter sets
# ---------------------------------------------------------------------------------------------

def test_default_params_file_is_the_references_byte_for_byte(ref, tmp_path):
    k = ref.keygen(seed=1)  # the reference's default 128-bit set
    try:
        k.save_params(str(tmp_path / "ref.txt"))
    finally:
        k.free()
    tb.save_params(str(tmp_path / "ours.txt"), tb.default_params())
    assert read(tmp_path / "ours.txt") == read(tmp_path / "ref.txt")
    p = tb.load_params(str(tmp_path / "ref.txt"))
    assert (p.n, p.N, p.k, p.l, p.Bgbit, p.ks_t, p.ks_basebit) == (630, 1024, 1, 3, 7, 8, 2)
    # reals are stored with 8 decimals, so a loaded stdev is the rounded value
    assert p.ks_stdev == pytest.approx(0.00003052, abs=1e-12)


def test_params_round_trip_keeps_every_integer_field(tmp_path):
    for p in (tb.default_params(), tb.large_params(), tb.default_params(80)):
        tb.save_params(str(tmp_path / "p.txt"), p)
        q = tb.load_params(str(tmp_path / "p.txt"))
        for f in ("n", "N", "k", "l", "Bgbit", "ks_t", "ks_basebit"):
            assert getattr(q, f) == getattr(p, f)
        assert q.ks_stdev == pytest.approx(float("%.8f" % p.ks_stdev), abs=1e-12)


# ---------------------------------------------------------------------------------------------
# key sets: reference -> here
# ---------------------------------------------------------------------------------------------

def test_reference_secret_keyset_loads_bit_exact_and_saves_back_identically(ref_keys, tmp_path):
    src = str(tmp_path / "ref_sk.bin")
    ref_keys.save_secret_keyset(src)
    sk, ck = tb.load_secret_keyset(src)
    lk, tk, kk, bk = ref_keys.export()
    bsk, ksk = ck.export()
    mlk, mtk = sk.export()
    assert (bsk == bk).all() and (ksk == kk).all()
    assert (mlk == lk).all() and (mtk == tk).all()
    assert ck.params.n == SMALL["n"] and ck.params.ks_t == SMALL["ks_t"]
    tb.save_secret_keyset(str(tmp_path / "ours_sk.bin"), sk, ck)
    assert read(tmp_path / "ours_sk.bin") == read(src)


def test_reference_cloud_keyset_loads_and_saves_back_identically(ref_keys, tmp_path):
    src = str(tmp_path / "ref_ck.bin")
    ref_keys.save_cloud_keyset(src)
    ck = tb.load_cloud_keyset(src)
    _, _, kk, bk = ref_keys.export()
    bsk, ksk = ck.export()
    assert (bsk == bk).all() and (ksk == kk).all()
    tb.save_cloud_keyset(str(tmp_path / "ours_ck.bin"), ck)
    assert read(tmp_path / "ours_ck.bin") == read(src)


def test_reference_keys_from_file_decrypt_reference_ciphertexts(ref_keys, tmp_path):
    ref_keys.save_secret_keyset(str(tmp_path / "sk.bin"))
    sk, _ = tb.load_secret_keyset(str(tmp_path / "sk.bin"))
    bits = np.random.default_rng(3).integers(0, 2, 64)
    got, _ = sk.decrypt(ref_keys.encrypt(bits))
    assert (got == bits).all()


# ---------------------------------------------------------------------------------------------
# key sets: here -> reference
# ---------------------------------------------------------------------------------------------

def test_our_secret_keyset_loads_in_the_reference_and_evaluates_gates(ref, tmp_path):
    p = small_params()
    sk, ck = tb.keygen(p, seed=2027)
    path = str(tmp_path / "ours_sk.bin")
    tb.save_secret_keyset(path, sk, ck)
    rk = ref.load_secret_keyset(path)
    try:
        lk, tk, kk, bk = rk.export()
        bsk, ksk = ck.export()
        mlk, mtk = sk.export()
        assert (bk == bsk).all() and (kk == ksk).all() and (lk == mlk).all() and (tk == mtk).all()
        # the reference re-exports it byte for byte
        rk.save_secret_keyset(str(tmp_path / "again.bin"))
        assert read(tmp_path / "again.bin") == read(path)
        # and computes with it: our encryptions, the reference's NAND, our decryption
        rng = np.random.default_rng(9)
        a, b = rng.integers(0, 2, 16), rng.integers(0, 2, 16)
        ca, cb = sk.encrypt(a, seed=1), sk.encrypt(b, seed=2)
        out = rk.gate(0, ca, cb)
        got, _ = sk.decrypt(out)
        assert (got == 1 - (a & b)).all()
        assert (rk.decrypt(ca)[0] == a).all()
    finally:
        rk.free()


# ---------------------------------------------------------------------------------------------
# ciphertexts
# ---------------------------------------------------------------------------------------------

def test_ciphertext_files_both_ways(ref_keys, tmp_path):
    p = small_params()
    rng = np.random.default_rng(11)
    cts = rng.integers(-2**31, 2**31, (7, p.n + 1), dtype=np.int64).astype(np.int32)
    var = rng.random(7)
    ref_keys.save_ciphertexts(str(tmp_path / "ref.ct"), cts, var)
    got, gv = tb.load_ciphertexts(str(tmp_path / "ref.ct"), p, 7)
    assert (got == cts).all() and (gv == var).all()
    tb.save_ciphertexts(str(tmp_path / "ours.ct"), p, cts, var)
    assert read(tmp_path / "ours.ct") == read(tmp_path / "ref.ct")
    back, bv = ref_keys.load_ciphertexts(str(tmp_path / "ours.ct"), 7)
    assert (back == cts).all() and (bv == var).all()


# ---------------------------------------------------------------------------------------------
# the drop-in's FILE* functions, from a C client
# ---------------------------------------------------------------------------------------------

def test_dropin_file_functions_from_c(ref_keys, tmp_path):
    program = str(tmp_path / "dropin_io")
    libdir = os.path.join(ROOT, "tfhe_b200")
    subprocess.check_call(["gcc", "-std=c99", "-O2", "-I", os.path.join(ROOT, "include"),
                           os.path.join(ROOT, "tests", "c", "dropin_io.c"), "-o", program,
                           "-L", libdir, "-ltfhe_b200", "-Wl,-rpath," + libdir])
    bits = np.random.default_rng(5).integers(0, 2, 24)
    cts = ref_keys.encrypt(bits)
    ref_keys.save_secret_keyset(str(tmp_path / "sk.bin"))
    ref_keys.save_ciphertexts(str(tmp_path / "in.ct"), cts, np.full(len(cts), 2.0**-30))
    ref_keys.save_params(str(tmp_path / "ref_params.txt"))
    out = [str(tmp_path / x) for x in ("sk2.bin", "out.ct", "params.txt")]
    res = subprocess.run([program, str(tmp_path / "sk.bin"), str(tmp_path / "in.ct"), str(len(bits))] + out,
                         capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr
    assert res.stdout.strip() == "".join(map(str, bits))
    assert read(out[0]) == read(tmp_path / "sk.bin")
    assert read(out[1]) == read(tmp_path / "in.ct")
    assert read(out[2]) == read(tmp_path / "ref_params.txt")


# ---------------------------------------------------------------------------------------------
# malformed input: an error status, not a crash
# ---------------------------------------------------------------------------------------------

def test_malformed_files_are_rejected(tmp_path):
    p = tb.default_params()
    sk, ck = tb.keygen(small_params(), seed=1)
    with pytest.raises(TfhebError):
        tb.load_params(str(tmp_path / "missing.txt"))
    (tmp_path / "junk.txt").write_text("-----BEGIN LWEPARAMS-----\nn: 630\n-----END LWEPARAMS-----\n")
    with pytest.raises(TfhebError, match="GATEBOOTSPARAMS"):
        tb.load_params(str(tmp_path / "junk.txt"))
    tb.save_secret_keyset(str(tmp_path / "sk.bin"), sk, ck)
    data = read(tmp_path / "sk.bin")
    (tmp_path / "short.bin").write_bytes(data[: len(data) // 2])
    with pytest.raises(TfhebError, match="truncated"):
        tb.load_secret_keyset(str(tmp_path / "short.bin"))
    # a cloud key set where a secret key set is expected: the LWE key block is missing
    tb.save_cloud_keyset(str(tmp_path / "ck.bin"), ck)
    with pytest.raises(TfhebError, match="LWE key"):
        tb.load_secret_keyset(str(tmp_path / "ck.bin"))
    # ciphertext block with the wrong type id
    tb.save_params(str(tmp_path / "p.txt"), p)
    with pytest.raises(TfhebError, match="LWE sample"):
        tb.load_ciphertexts(str(tmp_path / "p.txt"), p, 1)
