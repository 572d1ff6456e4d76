"""GPU parity of the hot path against the oracle (and the reference, through its golden vectors),
called through the C ABI.  Bars:
  * keyswitch, extraction, decomposition, rotation, mod-switch: bit-exact;
  * FP64 external product: exact after rounding to Torus32 (|error| <= 1 unit);
  * split-FP32 external product: per-coefficient error against the exact int128 product stated in
    Torus32 units, bounded here by max < 2^16 and RMS < 2^13 units per CMUX step (the bootstrapping
    key noise alone contributes ~2^18.5 units RMS per step);
  * gates: decrypt to the plaintext truth table and to the reference's bits.
"""
import os

import numpy as np
import pytest

import tfhe_b200 as tb
from tfhe_oracle import DEFAULT, LARGE, torus_diff

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")

TRUTH = {0: lambda a, b, c: 1 - (a & b), 1: lambda a, b, c: a | b, 2: lambda a, b, c: a & b,
         3: lambda a, b, c: a ^ b, 4: lambda a, b, c: 1 - (a ^ b), 5: lambda a, b, c: 1 - (a | b),
         6: lambda a, b, c: (1 - a) & b, 7: lambda a, b, c: a & (1 - b), 8: lambda a, b, c: (1 - a) | b,
         9: lambda a, b, c: a | (1 - b), 10: lambda a, b, c: np.where(a == 1, b, c), 11: lambda a, b, c: 1 - a,
         12: lambda a, b, c: a}


def dev(a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.int32)).cuda()


def host(t):
    torch.cuda.synchronize()
    return t.cpu().numpy()


def pdict(p):
    return dict(n=p.n, N=p.N, k=p.k, l=p.l, Bgbit=p.Bgbit, ks_t=p.ks_t, ks_basebit=p.ks_basebit)


@pytest.fixture(scope="module")
def default_keys():
    p = tb.default_params()
    sk, ck = tb.keygen(p, seed=2026)
    ck.to_device(0)
    bsk, ksk = ck.export()
    return p, sk, ck, bsk, ksk


@pytest.fixture(scope="module")
def golden_small():
    g = np.load(os.path.join(GOLDEN, "gates_small.npz"))
    p = tb.make_params(*map(int, g["params"]))
    ck = tb.CloudKey.from_raw(p, g["bsk"], g["ksk"]).to_device(0)
    sk = tb.SecretKey.from_raw(p, g["lwe_key"], g["tlwe_key"])
    return g, p, sk, ck


# ---------------------------------------------------------------------------------------------
# keyswitch: bit-exact
# ---------------------------------------------------------------------------------------------

def test_keyswitch_bit_exact_vs_reference_golden(golden_small):
    g, p, sk, ck = golden_small
    x = g["ks_inputs"]
    out = torch.zeros((len(x), p.n + 1), dtype=torch.int32, device="cuda")
    ck.keyswitch_device(dev(x), out, len(x))
    assert (host(out) == g["ks_outputs"]).all()


def test_keyswitch_other_shape_bit_exact_vs_reference_golden():
    # t=4, basebit=3: only the general per-sample kernel serves it; the tiled and register-key
    # kernels are instantiated for t=8, basebit=2 and refuse
    g = np.load(os.path.join(GOLDEN, "keyswitch_t4b3.npz"))
    p = tb.make_params(*map(int, g["params"]))
    bsk = np.zeros((p.n, (p.k + 1) * p.l, p.k + 1, p.N), np.int32)  # not used by the keyswitch
    ck = tb.CloudKey.from_raw(p, bsk, g["ksk"]).to_device(0, precisions=(tb.FP64,))
    x = g["ks_inputs"]
    out = torch.zeros((len(x), p.n + 1), dtype=torch.int32, device="cuda")
    ck.keyswitch_device(dev(x), out, len(x))
    assert (host(out) == g["ks_outputs"]).all()
    for which in (2, 3, 4):
        with pytest.raises(tb.api.TfhebError, match="no tiled keyswitch"):
            ck.set_keyswitch_kernel(which)


@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_gates_with_other_keyswitch_shape(precision):
    # the whole gate pipeline on the per-sample keyswitch (t=4, basebit=3)
    p = tb.make_params(200, 1024, 1, 3, 7, 4, 3)
    sk, ck = tb.keygen(p, seed=43)
    ck.to_device(0)
    rng = np.random.default_rng(44)
    x, y = rng.integers(0, 2, 300), rng.integers(0, 2, 300)
    out = ck.gate(tb.api.XOR, sk.encrypt(x, seed=1), sk.encrypt(y, seed=2), precision=precision)
    got, _ = sk.decrypt(out)
    assert (got == (x ^ y)).all()


def test_keyswitch_bit_exact_vs_oracle_default(oracle, default_keys):
    p, sk, ck, bsk, ksk = default_keys
    rng = np.random.default_rng(1)
    x = rng.integers(-2**31, 2**31, (64, p.k * p.N + 1), dtype=np.int64).astype(np.int32)
    x[0] = 0
    x[1] = -1
    out = torch.zeros((64, p.n + 1), dtype=torch.int32, device="cuda")
    ck.keyswitch_device(dev(x), out, 64)
    got = host(out)
    want = oracle.keyswitch(pdict(p), ksk, x[:16])
    assert (got[:16] == want).all()


def _keyswitch_with(ck, p, x, which, fill):
    ck.set_keyswitch_kernel(which)
    try:
        out = torch.full((len(x), p.n + 1), fill, dtype=torch.int32, device="cuda")
        ck.keyswitch_device(dev(x), out, len(x))
        return host(out)
    finally:
        ck.set_keyswitch_kernel(0)


# batch sizes: 1 and 63 split the coefficient range over CTAs (atomic combination), 64/65/300 give
# full and ragged 64-sample tiles (256-sample tiles of the tensor-core kernel: 300 and 2100 end
# ragged), 2100 more tiles than one wave of CTAs
@pytest.mark.parametrize("count", [1, 63, 64, 65, 300, 2100])
def test_keyswitch_kernels_agree_bit_for_bit(oracle, default_keys, count):
    p, sk, ck, bsk, ksk = default_keys
    rng = np.random.default_rng(100 + count)
    x = rng.integers(-2**31, 2**31, (count, p.k * p.N + 1), dtype=np.int64).astype(np.int32)
    x[0] = -1
    per_sample = _keyswitch_with(ck, p, x, 1, 0)
    tiled = _keyswitch_with(ck, p, x, 2, -7)  # garbage in the output rows must not leak through
    regkey = _keyswitch_with(ck, p, x, 3, 13)
    tensor_core = _keyswitch_with(ck, p, x, 4, 99)
    assert (tiled == per_sample).all()
    assert (regkey == per_sample).all()
    assert (tensor_core == per_sample).all()
    pick = sorted({0, count - 1, count // 2})
    assert (tiled[pick] == oracle.keyswitch(pdict(p), ksk, x[pick])).all()


def test_keyswitch_tiled_large_params_bit_exact(oracle, large_keys):
    p, sk, ck, bsk, ksk = large_keys
    rng = np.random.default_rng(7)
    x = rng.integers(-2**31, 2**31, (130, p.k * p.N + 1), dtype=np.int64).astype(np.int32)
    tiled = _keyswitch_with(ck, p, x, 2, 5)
    assert (tiled == _keyswitch_with(ck, p, x, 1, 0)).all()
    assert (tiled == _keyswitch_with(ck, p, x, 3, -3)).all()
    assert (tiled == _keyswitch_with(ck, p, x, 4, 17)).all()
    assert (tiled[[0, 129]] == oracle.keyswitch(pdict(p), ksk, x[[0, 129]])).all()


# the tensor-core kernel's tile edges (256 samples per CTA: 255 / 256 / 257; those split the
# coefficient range over CTAs and combine with atomic adds) and 7421 samples, 29 tiles x 10 column
# groups = 290 CTAs, which its wave model runs with one coefficient range per CTA (plain stores);
# every kernel must agree bit for bit
@pytest.mark.parametrize("count", [255, 256, 257, 7421])
def test_keyswitch_tensor_core_tile_edges(oracle, default_keys, count):
    p, sk, ck, bsk, ksk = default_keys
    rng = np.random.default_rng(300 + count)
    x = rng.integers(-2**31, 2**31, (count, p.k * p.N + 1), dtype=np.int64).astype(np.int32)
    x[-1] = 0
    tensor_core = _keyswitch_with(ck, p, x, 4, 11)
    assert (tensor_core == _keyswitch_with(ck, p, x, 3, -11)).all()
    assert (tensor_core == _keyswitch_with(ck, p, x, 0, 5)).all()  # the default is the tensor-core kernel
    pick = sorted({0, 255 % count, count - 1})
    assert (tensor_core[pick] == oracle.keyswitch(pdict(p), ksk, x[pick])).all()


def test_keyswitch_tensor_core_80bit_partial_column_group(oracle):
    # n = 500: 501 output columns, the last 64-column group holds 53 of them
    p = tb.default_params(80)
    sk, ck = tb.keygen(p, seed=80)
    ck.to_device(0, precisions=(tb.FP64,))
    bsk, ksk = ck.export()
    rng = np.random.default_rng(81)
    x = rng.integers(-2**31, 2**31, (300, p.k * p.N + 1), dtype=np.int64).astype(np.int32)
    tensor_core = _keyswitch_with(ck, p, x, 4, 9)
    assert (tensor_core == _keyswitch_with(ck, p, x, 1, 0)).all()
    assert (tensor_core[[0, 299]] == oracle.keyswitch(pdict(p), ksk, x[[0, 299]])).all()


# ---------------------------------------------------------------------------------------------
# one CMUX step = rotation + decomposition + external product: exact (FP64) / bounded (split)
# ---------------------------------------------------------------------------------------------

def cmux_errors(oracle, p, ck, bsk, precision, count=6, seed=3):
    rng = np.random.default_rng(seed)
    acc = rng.integers(-2**31, 2**31, (count, p.k + 1, p.N), dtype=np.int64).astype(np.int32)
    a = rng.integers(1, 2 * p.N, count).astype(np.int32)
    d_acc = dev(acc)
    ck.blind_rotate_device(dev(a.reshape(count, 1)), d_acc, count, 1, precision=precision)
    got = host(d_acc)
    errs = []
    for gi in range(count):
        want = oracle.cmux_step(pdict(p), bsk[0], a[gi], acc[gi].reshape(-1))
        errs.append(torus_diff(got[gi].reshape(-1), want))
    return np.concatenate(errs)


@pytest.fixture(scope="module")
def large_keys():
    p = tb.large_params()
    sk, ck = tb.keygen(p, seed=4048)
    ck.to_device(0)
    bsk, ksk = ck.export()
    return p, sk, ck, bsk, ksk


def test_cmux_step_fp64_exact(oracle, default_keys):
    p, sk, ck, bsk, ksk = default_keys
    err = cmux_errors(oracle, p, ck, bsk, tb.FP64)
    assert np.abs(err).max() <= 1


def test_cmux_step_fp64_exact_large_ring(oracle, large_keys):
    p, sk, ck, bsk, ksk = large_keys
    err = cmux_errors(oracle, p, ck, bsk, tb.FP64, count=3)
    assert np.abs(err).max() <= 1


@pytest.mark.parametrize("ring", ["default", "large"])
def test_cmux_step_split_fp32_error_bound(oracle, request, ring):
    # per-coefficient error of one CMUX step against the exact int128 product, in Torus32 units;
    # per-step bootstrapping-key noise is ~2^18.5 (N=1024) / ~2^20 (N=2048) units rms
    p, sk, ck, bsk, ksk = request.getfixturevalue(f"{ring}_keys")
    err = cmux_errors(oracle, p, ck, bsk, tb.SPLIT_FP32, count=4)
    rms = float(np.sqrt((err.astype(np.float64) ** 2).mean()))
    print(f"split-FP32 CMUX error vs exact (N={p.N}): max {np.abs(err).max()} units, rms {rms:.1f} units")
    # the low limb carries 2^S with S = 24 (N=1024) / 26 (N=2048): its FP32 error scales with 2^S
    scale = 1 if p.N == 1024 else 4
    assert np.abs(err).max() < scale * 2**17
    assert rms < scale * 2**14


@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_cmux_step_packed_and_digit_parallel_kernels(oracle, default_keys, precision):
    # 1040 accumulators (more than one wave at 7 per CTA) run on the packed kernel; 6 of them again
    # alone run on the digit-parallel kernel: the same bits, and samples of the large batch within
    # the single-step bounds of the exact oracle
    p, sk, ck, bsk, ksk = default_keys
    rng = np.random.default_rng(11 + precision)
    count = 1040
    acc = rng.integers(-2**31, 2**31, (count, p.k + 1, p.N), dtype=np.int64).astype(np.int32)
    a = rng.integers(1, 2 * p.N, count).astype(np.int32)
    d_acc = dev(acc)
    ck.blind_rotate_device(dev(a.reshape(count, 1)), d_acc, count, 1, precision=precision)
    big = host(d_acc)
    d_small = dev(acc[:6])
    ck.blind_rotate_device(dev(a[:6].reshape(6, 1)), d_small, 6, 1, precision=precision)
    assert (host(d_small) == big[:6]).all()
    for gi in (0, 517, count - 1):
        want = oracle.cmux_step(pdict(p), bsk[0], a[gi], acc[gi].reshape(-1))
        err = torus_diff(big[gi].reshape(-1), want)
        assert np.abs(err).max() <= (1 if precision == tb.FP64 else 2**17)


def test_blind_rotate_many_steps_fp64_matches_oracle(oracle, default_keys):
    # 40 consecutive CMUX steps from a random accumulator: FP64 products round to the exact value,
    # so the GPU accumulator equals the oracle's almost everywhere (a rare +-1 can flip a digit).
    p, sk, ck, bsk, ksk = default_keys
    rng = np.random.default_rng(5)
    steps = 40
    acc = rng.integers(-2**31, 2**31, (1, p.k + 1, p.N), dtype=np.int64).astype(np.int32)
    bara = rng.integers(0, 2 * p.N, (1, steps)).astype(np.int32)
    d_acc = dev(acc)
    ck.blind_rotate_device(dev(bara), d_acc, 1, steps, precision=tb.FP64)
    got = host(d_acc).reshape(-1)
    sub = dict(pdict(p), n=steps)
    want = oracle.blind_rotate(sub, bsk[:steps], bara[0], acc.reshape(-1))
    assert (got == want).mean() > 0.99


# ---------------------------------------------------------------------------------------------
# gates
# ---------------------------------------------------------------------------------------------

@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_gates_golden_small_match_reference_bits(golden_small, precision):
    g, p, sk, ck = golden_small
    codes = g["gate_codes"]
    for code in np.unique(codes):
        sel = codes == code
        out = ck.gate(int(code), g["ca"][sel], g["cb"][sel], g["cc"][sel] if code == 10 else None,
                      precision=precision)
        bits, _ = sk.decrypt(out)
        assert (bits == g["out_bits"][sel]).all(), f"gate {tb.api.GATE_NAMES[code]}"


@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_all_gates_default_params_truth_tables(default_keys, precision):
    p, sk, ck, bsk, ksk = default_keys
    rng = np.random.default_rng(7 + precision)
    G = 96
    a, b, c = rng.integers(0, 2, (3, G))
    ca, cb, cc = sk.encrypt(a, seed=1), sk.encrypt(b, seed=2), sk.encrypt(c, seed=3)
    for code in range(13):
        out = ck.gate(code, ca, cb, cc if code == 10 else None, precision=precision)
        bits, _ = sk.decrypt(out)
        assert (bits == TRUTH[code](a, b, c)).all(), f"gate {tb.api.GATE_NAMES[code]}"


@pytest.fixture(scope="module")
def keys80():
    p = tb.default_params(80)
    sk, ck = tb.keygen(p, seed=80)
    ck.to_device(0)
    return p, sk, ck


@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_80bit_params_all_gates_and_a_4096_batch(keys80, precision):
    # the reference's 80-bit set (n=500, l=2, Bgbit=10): every gate's truth table, then 4096 NANDs
    p, sk, ck = keys80
    assert (p.n, p.l, p.Bgbit) == (500, 2, 10)
    rng = np.random.default_rng(80 + precision)
    a, b, c = rng.integers(0, 2, (3, 64))
    ca, cb, cc = sk.encrypt(a, seed=1), sk.encrypt(b, seed=2), sk.encrypt(c, seed=3)
    for code in range(13):
        bits, _ = sk.decrypt(ck.gate(code, ca, cb, cc if code == 10 else None, precision=precision))
        assert (bits == TRUTH[code](a, b, c)).all(), f"gate {tb.api.GATE_NAMES[code]}"
    x, y = rng.integers(0, 2, (2, 4096))
    ex, ey = sk.encrypt(x, seed=4), sk.encrypt(y, seed=5)
    out = ck.gate(tb.api.NAND, ex, ey, precision=precision)
    bits, ph = sk.decrypt(out)
    assert (bits == 1 - (x & y)).all()
    # 64 gates run one bootstrap per CTA (the digit-parallel kernel), 4096 run packed: same bits
    assert (ck.gate(tb.api.NAND, ex[:64], ey[:64], precision=precision) == out[:64]).all()
    # outputs sit at +-1/8 = +-2^29 Torus32 units; a decryption error needs |noise| > 2^29.  With
    # 10-bit digits the split form's low limb carries S = 27 bits, so its FP32 error adds to the
    # noise; both forms keep the rms far below the margin.
    err = (ph.astype(np.int64) - np.where(bits == 1, 2**29, -2**29) + 2**31) % 2**32 - 2**31
    rms = float(np.sqrt((err.astype(np.float64) ** 2).mean()))
    print(f"80-bit set, precision {precision}: output noise rms 2^{np.log2(rms):.2f}, max 2^{np.log2(np.abs(err).max()):.2f}")
    # measured: FP64 rms 2^24.1 (the reference's precision), split 2^26.0 (the low limb's FP32 error)
    assert rms < (2**25 if precision == tb.FP64 else 2**26.5)


@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_nand_batch_4096_decrypts_and_noise_matches_reference(default_keys, golden_dir, precision):
    # 4096 NANDs in one batch; output noise variance (phase - (+-1/8)) against the reference's
    # spqlios build measured on 8000 gates (tests/golden/noise_default.npz): within 10%.
    p, sk, ck, bsk, ksk = default_keys
    rng = np.random.default_rng(11 + precision)
    G = 4096
    a, b = rng.integers(0, 2, (2, G))
    out = ck.gate(tb.api.NAND, sk.encrypt(a, seed=21), sk.encrypt(b, seed=22), precision=precision)
    bits, ph = sk.decrypt(out)
    truth = 1 - (a & b)
    assert (bits == truth).all()
    err = torus_diff(ph, np.where(truth == 1, 1 << 29, -(1 << 29))).astype(np.float64)
    ref = np.load(os.path.join(golden_dir, "noise_default.npz"))
    ratio = err.var() / float(ref["err_var"])
    print(f"precision {precision}: noise var {err.var():.4g} vs reference {float(ref['err_var']):.4g} "
          f"(ratio {ratio:.3f}), mean {err.mean():.4g}")
    assert 0.9 < ratio < 1.1


@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_mux_large_ring_n2048(large_keys, precision):
    p, sk, ck, bsk, ksk = large_keys
    rng = np.random.default_rng(13)
    G = 64
    a, b, c = rng.integers(0, 2, (3, G))
    out = ck.gate(tb.api.MUX, sk.encrypt(a, seed=1), sk.encrypt(b, seed=2), sk.encrypt(c, seed=3),
                  precision=precision)
    bits, _ = sk.decrypt(out)
    assert (bits == np.where(a == 1, b, c)).all()


def test_bootstrap_woks_device_matches_oracle_phase(oracle, default_keys):
    # tfhe_bootstrap_woKS_FFT on the GPU vs the exact oracle: same message, phases within noise.
    p, sk, ck, bsk, ksk = default_keys
    rng = np.random.default_rng(17)
    a, b = rng.integers(0, 2, (2, 4))
    x = oracle.gate_prologue(p.n, 0, sk.encrypt(a, seed=3), sk.encrypt(b, seed=4))
    mu = oracle.modswitch_to(1, 8)
    out = torch.zeros((4, p.k * p.N + 1), dtype=torch.int32, device="cuda")
    ck.bootstrap_woks_device(dev(x), out, 4, mu, precision=tb.FP64)
    got = host(out)
    want = oracle.bootstrap_woks(pdict(p), bsk, mu, x[:2])
    lk, tk = sk.export()
    d = torus_diff(oracle.phase(tk, got[:2]), oracle.phase(tk, want))
    assert np.abs(d).max() < 2**24
    assert ((oracle.phase(tk, got) > 0) == (1 - (a & b) == 1)).all()
