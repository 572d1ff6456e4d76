"""Pins the C oracle to the reference: every building block against golden vectors produced by the
reference library itself (tests/golden/make_golden.py), and, when the reference build is present
in this checkout (oracle/_ref), against live reference calls on identical inputs."""
import os

import numpy as np
import pytest

from tfhe_oracle import torus_diff
from tfhe_ref import RefLib


def load(golden_dir, name):
    return np.load(os.path.join(golden_dir, name))


def test_modswitch_known_answers(oracle, golden_dir):
    g = load(golden_dir, "numerics.npz")
    for mi, m in enumerate(g["msizes"]):
        got = np.array([oracle.modswitch_from(p, m) for p in g["phases"]], np.int32)
        assert (got == g["ms_from"][mi]).all(), f"modSwitchFromTorus32 Msize={m}"
        got = np.array([oracle.modswitch_to(u, m) for u in g["mus"]], np.int32)
        assert (got == g["ms_to"][mi]).all(), f"modSwitchToTorus32 Msize={m}"


@pytest.mark.parametrize("N,l,bgbit", [(1024, 3, 7), (2048, 3, 8), (1024, 2, 10)])
def test_decomposition_golden(oracle, golden_dir, N, l, bgbit):
    g = load(golden_dir, "decomposition.npz")
    tag = f"N{N}_l{l}_b{bgbit}"
    for poly, digits in zip(g[f"{tag}_polys"], g[f"{tag}_digits"]):
        assert (oracle.decompose(N, l, bgbit, poly) == digits).all()


def test_decomposition_recomposition_bound(oracle):
    # tgsw_test.cpp:581-611: |sum_p d_p h_p - c| <= 2^(32 - l*Bgbit) in Torus32 units (the offset
    # centres the digits but carries no half-unit rounding term, so the last digit truncates)
    rng = np.random.default_rng(3)
    for (N, l, bgbit) in [(1024, 3, 7), (2048, 3, 8)]:
        poly = rng.integers(-2**31, 2**31, N, dtype=np.int64).astype(np.int32)
        d = oracle.decompose(N, l, bgbit, poly).astype(np.int64)
        recomposed = sum(d[p] << (32 - (p + 1) * bgbit) for p in range(l))
        err = torus_diff(recomposed, poly)
        assert np.abs(err).max() <= 1 << (32 - l * bgbit)
        assert d.min() >= -(1 << (bgbit - 1)) and d.max() < (1 << (bgbit - 1))


@pytest.mark.parametrize("N", [1024, 2048])
def test_rotations_golden(oracle, golden_dir, N):
    g = load(golden_dir, "rotations.npz")
    poly = g[f"N{N}_poly"]
    for i, a in enumerate(g[f"N{N}_a"]):
        assert (oracle.rotate(N, a, False, poly) == g[f"N{N}_xai"][i]).all()
        assert (oracle.rotate(N, a, True, poly) == g[f"N{N}_xai_minus_one"][i]).all()


@pytest.mark.parametrize("N,k", [(1024, 1), (2048, 1), (512, 2)])
def test_extraction_golden(oracle, golden_dir, N, k):
    g = load(golden_dir, "extraction.npz")
    assert (oracle.extract(N, k, g[f"N{N}_k{k}_tlwe"]) == g[f"N{N}_k{k}_lwe"]).all()


@pytest.mark.parametrize("N", [512, 1024, 2048])
def test_exact_product_golden(oracle, golden_dir, N):
    g = load(golden_dir, "products.npz")
    for i in range(2):
        ip, tp = g[f"N{N}_int"][i], g[f"N{N}_torus"][i]
        got = oracle.negacyclic_mult(N, ip, tp)
        assert (got == g[f"N{N}_naive"][i]).all()
        assert (got == g[f"N{N}_karatsuba"][i]).all()
        if N == 1024:  # test-multiplication.cpp:66-77: |FFT - naive| <= 1 unit
            assert np.abs(torus_diff(g[f"N{N}_fft"][i], got)).max() <= 1


def test_wide_product_reduces_to_wrapping_product(oracle):
    rng = np.random.default_rng(11)
    N = 256
    ip = rng.integers(-64, 64, N).astype(np.int32)
    tp = rng.integers(-2**31, 2**31, N, dtype=np.int64).astype(np.int32)
    wide = oracle.negacyclic_mult_wide(N, ip, tp)
    red = np.array([((int(w) + 2**31) % 2**32) - 2**31 for w in wide], np.int64)
    assert (red == oracle.negacyclic_mult(N, ip, tp)).all()


def small_keys(golden_dir):
    g = load(golden_dir, "gates_small.npz")
    p = dict(zip(("n", "N", "k", "l", "Bgbit", "ks_t", "ks_basebit"), map(int, g["params"])))
    return g, p


def test_keyswitch_golden_bit_exact(oracle, golden_dir):
    g, p = small_keys(golden_dir)
    out = oracle.keyswitch(p, g["ksk"], g["ks_inputs"])
    assert (out == g["ks_outputs"]).all()


def test_keyswitch_golden_other_shape_bit_exact(oracle, golden_dir):
    # t=4, basebit=3 (the general keyswitch shape, tests/golden/keyswitch_t4b3.npz)
    g = np.load(os.path.join(golden_dir, "keyswitch_t4b3.npz"))
    p = dict(zip(("n", "N", "k", "l", "Bgbit", "ks_t", "ks_basebit"), map(int, g["params"])))
    assert g["ksk"].shape == (p["k"] * p["N"], 4, 8, p["n"] + 1)
    out = oracle.keyswitch(p, g["ksk"], g["ks_inputs"])
    assert (out == g["ks_outputs"]).all()


def test_gates_golden_decrypt_and_phase(oracle, golden_dir):
    g, p = small_keys(golden_dir)
    codes = g["gate_codes"]
    for code in np.unique(codes):
        sel = codes == code
        out = oracle.gate(p, g["bsk"], g["ksk"], int(code), g["ca"][sel], g["cb"][sel], g["cc"][sel])
        ph = oracle.phase(g["lwe_key"], out)
        assert ((ph > 0).astype(np.int32) == g["out_bits"][sel]).all(), f"gate {code}"
        # both outputs sit within the 1/16 decryption margin around +-1/8
        mu = np.where(g["out_bits"][sel] == 1, 1 << 29, -(1 << 29))
        assert np.abs(torus_diff(ph, mu)).max() < 1 << 28
        if code in (11, 12):  # NOT / COPY are bootstrap-free and bit-exact
            assert (out == g["outputs"][sel]).all()


def test_bootstrap_phase_matches_reference(oracle, golden_dir):
    # Before the keyswitch, compare phases under the extracted key.  The reference's products
    # truncate and the oracle's are exact; the first +-1 difference flips a gadget digit, after which
    # the two accumulators carry different masks and therefore different (equally distributed)
    # bootstrapping-key noise: per step sqrt(N*kpl)*rms(digit)*sigma_bk ~ 2^18.5 Torus32 units, so
    # over n=16 steps the two phases differ by ~2^21 rms.  Bound: 2^24 (6 sigma), far below 1/16.
    ref = RefLib.load()
    if ref is None:
        pytest.skip("reference build (oracle/_ref) not present")
    g, p = small_keys(golden_dir)
    keys = ref.keygen(custom=p, seed=77)  # same seed as the fixture: identical keys
    try:
        lk, tk, _, bsk = keys.export(ksk=False)
        assert (lk == g["lwe_key"]).all() and (bsk == g["bsk"]).all()
        x = oracle.gate_prologue(p["n"], 0, g["ca"][:8], g["cb"][:8])
        mu = oracle.modswitch_to(1, 8)
        got = oracle.bootstrap_woks(p, bsk, mu, x)
        want = keys.bootstrap_woks(mu, x)
        d = torus_diff(oracle.phase(tk, got), oracle.phase(tk, want))
        assert np.abs(d).max() < 2**24
    finally:
        keys.free()


def test_gate_truth_tables(oracle, golden_dir):
    g, p = small_keys(golden_dir)
    a, b, c = g["bits"]
    truth = {0: 1 - (a & b), 1: a | b, 2: a & b, 3: a ^ b, 4: 1 - (a ^ b), 5: 1 - (a | b),
             6: (1 - a) & b, 7: a & (1 - b), 8: (1 - a) | b, 9: a | (1 - b), 10: np.where(a == 1, b, c),
             11: 1 - a, 12: a}
    codes = g["gate_codes"]
    for code, t in truth.items():
        sel = codes == code
        assert (g["out_bits"][sel] == t[sel]).all(), f"reference gate {code} truth table"


ref_live = pytest.mark.skipif(not RefLib.available(), reason="reference build (oracle/_ref) not present")


@ref_live
def test_live_external_product_within_one_unit(oracle):
    ref = RefLib.load()
    keys = ref.keygen(custom=None, seed=5)
    try:
        p = keys.params()
        _, _, _, bsk = keys.export(ksk=False)
        rng = np.random.default_rng(8)
        for i in (0, 17, 629):
            acc = rng.integers(-2**31, 2**31, (p["k"] + 1) * p["N"], dtype=np.int64).astype(np.int32)
            got = oracle.external_product(p, bsk[i], acc)
            want = keys.extern_mul(i, acc)
            assert np.abs(torus_diff(got, want)).max() <= 1
    finally:
        keys.free()


@ref_live
def test_live_keyswitch_default_params_bit_exact(oracle):
    ref = RefLib.load()
    keys = ref.keygen(custom=None, seed=6)
    try:
        p = keys.params()
        _, _, ksk, _ = keys.export(bsk=False)
        rng = np.random.default_rng(9)
        x = rng.integers(-2**31, 2**31, (6, p["k"] * p["N"] + 1), dtype=np.int64).astype(np.int32)
        assert (oracle.keyswitch(p, ksk, x) == keys.keyswitch(x)).all()
    finally:
        keys.free()
