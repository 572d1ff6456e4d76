"""CPU-only checks of the product library: it loads without a GPU, exports every symbol its headers
declare, and its host-side key material is valid when evaluated by the independent oracle."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import tfhe_b200 as tb
from tfhe_oracle import torus_diff

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_functions(path):
    text = open(path).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    names = set()
    for m in re.finditer(r"([A-Za-z_][A-Za-z0-9_]*)\s*\(", text):
        name = m.group(1)
        if name in ("if", "for", "while", "sizeof", "return", "defined"):
            continue
        # a declaration: preceded by a type on the same statement
        start = text.rfind(";", 0, m.start())
        stmt = text[start + 1:m.start()]
        if "typedef" in stmt or "#define" in stmt or "struct" in stmt.split()[-1:] or not stmt.strip():
            continue
        names.add(name)
    return names


@pytest.mark.parametrize("header", ["tfhe_b200.h", "tfhe.h"])
def test_library_exports_every_declared_symbol(header):
    L = tb.api.lib()
    missing = [f for f in sorted(header_functions(os.path.join(ROOT, "include", header))) if not hasattr(L, f)]
    assert not missing, f"symbols declared in include/{header} but not exported: {missing}"


def test_status_codes_without_gpu_work():
    p = tb.default_params()
    assert (p.n, p.N, p.k, p.l, p.Bgbit, p.ks_t, p.ks_basebit) == (630, 1024, 1, 3, 7, 8, 2)
    assert abs(p.ks_stdev - 2**-15) < 1e-20 and abs(p.bk_stdev - 2**-25) < 1e-20
    p80 = tb.default_params(80)
    assert (p80.n, p80.l, p80.Bgbit) == (500, 2, 10)
    with pytest.raises(tb.api.TfhebError):
        tb.default_params(129)
    q = tb.large_params()
    assert (q.n, q.N, q.l, q.Bgbit) == (800, 2048, 3, 8)


def test_encrypt_decrypt_roundtrip():
    sk, ck = tb.keygen(tb.default_params(), seed=11)
    bits = np.random.default_rng(1).integers(0, 2, 500)
    ct = sk.encrypt(bits, seed=2)
    got, ph = sk.decrypt(ct)
    assert (got == bits).all()
    err = torus_diff(ph, np.where(bits == 1, 1 << 29, -(1 << 29)))
    assert np.abs(err).max() < 2**20  # fresh noise stdev 2^-15 = 2^17 units


@pytest.mark.parametrize("N", [128, 512, 1024, 2048])
def test_fft_slot_order_is_a_permutation_matching_the_stage_model(N):
    sf = tb.fft_slot_order(N)
    M = N // 2
    assert sorted(sf.flatten().tolist()) == list(range(M))
    # model: positions of the last stage, mixed-radix digit reversal (see tfhe_b200/csrc/fft.cuh)
    plans = {64: [8, 8], 256: [8, 8, 4], 512: [8, 8, 8], 1024: [8, 8, 8, 2]}[M]
    lens = [M]
    for r in plans:
        lens.append(lens[-1] // r)
    NT = M // 8
    rl = plans[-1]
    for t in range(0, NT, max(1, NT // 7)):
        for reg in range(8):
            c, n2 = divmod(reg, rl)
            L = lens[-2]
            st = L // rl
            b = t + NT * c
            pos = (b // st) * L + (b % st) + st * n2
            k, mul = 0, 1
            for s, r in enumerate(plans):
                k += ((pos // lens[s + 1]) % r) * mul
                mul *= r
            assert sf[reg, t] == k


@pytest.fixture(scope="module")
def small_engine_keys():
    p = tb.make_params(16, 1024, 1, 3, 7, 8, 2)
    sk, ck = tb.keygen(p, seed=5)
    bsk, ksk = ck.export()
    lk, tk = sk.export()
    return p, sk, ck, bsk, ksk, lk, tk


def test_engine_keys_evaluate_correctly_in_the_oracle(oracle, small_engine_keys):
    # The engine's host key generation, evaluated by the independent exact oracle: gates decrypt right.
    p, sk, ck, bsk, ksk, lk, tk = small_engine_keys
    pd = dict(n=p.n, N=p.N, k=p.k, l=p.l, Bgbit=p.Bgbit, ks_t=p.ks_t, ks_basebit=p.ks_basebit)
    rng = np.random.default_rng(4)
    a, b = rng.integers(0, 2, (2, 6))
    ca, cb = sk.encrypt(a, seed=8), sk.encrypt(b, seed=9)
    for code, fn in ((0, lambda x, y: 1 - (x & y)), (3, lambda x, y: x ^ y)):
        out = oracle.gate(pd, bsk, ksk, code, ca, cb)
        got, _ = sk.decrypt(out)
        assert (got == fn(a, b)).all()


def test_engine_bsk_rows_encrypt_key_times_gadget(oracle, small_engine_keys):
    p, sk, ck, bsk, ksk, lk, tk = small_engine_keys
    N = p.N
    for i in (0, 7, 15):
        for q in range(p.l):
            row = bsk[i, p.l + q]  # body block: phase = e + s_i * h_q at coefficient 0
            ph = (row[1].astype(np.int64) - oracle.negacyclic_mult(N, tk, row[0])) % 2**32
            want = np.zeros(N, np.int64)
            want[0] = (int(lk[i]) << (32 - (q + 1) * p.Bgbit)) % 2**32
            assert np.abs(torus_diff(ph, want)).max() < 2**12  # bk noise stdev 2^-25 = 2^7 units


def test_dropin_header_compiles_as_c_and_cxx(tmp_path):
    src = tmp_path / "prog.c"
    src.write_text(
        '#include "tfhe.h"\n#include "tfhe_b200.h"\n'
        "int main(void){TFheGateBootstrappingParameterSet*p=new_default_gate_bootstrapping_parameters(110);"
        "return p->in_out_params->n == 630 ? 0 : 1;}\n")
    inc = os.path.join(ROOT, "include")
    for compiler, flags in (("gcc", ["-std=c99"]), ("g++", ["-x", "c++"])):
        subprocess.check_call([compiler, *flags, "-I", inc, "-c", str(src), "-o", str(tmp_path / "prog.o")])


def test_bench_script_parses_and_lists_its_workloads():
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = subprocess.run([sys.executable, os.path.join(root, "bench.py"), "--help"], capture_output=True, text=True,
                         timeout=120)
    assert res.returncode == 0, res.stderr
    for w in ("netlist", "mux2048", "errors", "keyswitch"):
        assert w in res.stdout


def test_blind_rotation_defaults_listed_first():
    # the first candidate of each parameter set is the default until tfheb_autotune measures
    # otherwise: split G=7 with a 12-half-row ring (two transforms per thread) and FP64 G=4 D=5 at
    # N=1024 (l=3); at N=2048 split G=3 with a 6-deep ring (two transforms per thread, the rotated
    # words parked in TMEM), FP64 G=2
    want = {(1024, tb.SPLIT_FP32): (7, 12), (1024, tb.FP64): (4, 5),
            (2048, tb.SPLIT_FP32): (3, 6), (2048, tb.FP64): (2, 3)}
    for (N, prec), gd in want.items():
        G, D = tb.api.br_variants(N, prec)
        assert len(G) >= 2 and (int(G[0]), int(D[0])) == gd
        assert (G >= 1).all() and (D >= 3).all()


def test_key_without_keyswitching_key_serves_rotations_only(tmp_path):
    # a cloud key imported with a null keyswitching key (what the drop-in builds from caller-made
    # TGSW samples): importing works, saving it in the reference's format is refused
    p = tb.make_params(8, 1024, 1, 3, 7, 8, 2)
    bsk = np.zeros((p.n, (p.k + 1) * p.l, p.k + 1, p.N), np.int32)
    L = tb.api.lib()
    h = ctypes.c_void_p()
    assert L.tfheb_cloud_key_import(ctypes.byref(p), bsk.ctypes.data_as(ctypes.c_void_p), None, ctypes.byref(h)) == 0
    try:
        path = str(tmp_path / "ck.key")
        assert L.tfheb_cloud_key_save(h, path.encode()) == 1
        assert b"keyswitching key" in L.tfheb_last_error()
    finally:
        L.tfheb_cloud_key_free(h)


def test_fft_plans_listed_per_variant():
    # plan 0: one transform per thread; plan 1: two per thread on packed f32x2 with the spectra in
    # tensor memory (split-FP32 only)
    for N, prec in ((1024, tb.SPLIT_FP32), (2048, tb.SPLIT_FP32), (1024, tb.FP64), (2048, tb.FP64)):
        p = tb.default_params() if N == 1024 else tb.large_params()
        sk, ck = tb.keygen(tb.make_params(8, N, 1, 3, p.Bgbit, 8, 2), seed=1)
        G, D = ck.br_variants(prec)
        plans = ck.br_plans(prec)
        assert len(plans) == len(G)
        assert set(plans.tolist()) == ({0, 1} if prec == tb.SPLIT_FP32 else {0})
