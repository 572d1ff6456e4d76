"""Bit-exact GPU pins of the integer steps of the bootstrap, through the C ABI.

The blind rotation's floating-point products round to the exact integer whenever their error stays
below half a unit, and then every step of tfhe_bootstrap_woKS_FFT (lwe-bootstrapping-functions-fft.cpp:
169-200) is integer arithmetic with one right answer:
  * the gate prologue and modSwitchFromTorus32 (numeric-functions.cpp:59-65) of every a_i and of b;
  * the test vector X^{2N-barb} * [mu..mu] (lwe-bootstrapping-functions-fft.cpp:142-145);
  * (X^a - 1) * acc (tlwe-functions.cpp:202-206) and the gadget decomposition (tgsw-functions.cpp:
    297-410);
  * sample extraction at index 0 (lwe.cpp:41-53), mask and body.
Two families of inputs make the products exact, so the GPU output must equal the oracle (exact
integer products) bit for bit:
  * zero rotation: every a_i = 0, so every bara_i = 0 and every step adds an exact zero; the output
    is the extraction of the rotated test vector, on the real keys of both rings and both forms;
  * coarse bootstrapping keys: every key coefficient is h * 2^S with |h| <= 2 (S the split shift),
    so the split form's low limb is exactly zero and every product sum stays below 2^20 units of
    2^S: both forms round exactly, for all n steps, with non-zero masks in the accumulator.  The
    inputs' a_i and b come from the reference's mod-switch golden vectors (tests/golden/numerics.npz),
    whose values the oracle's mod-switch reproduces exactly, checked here too.
A small-magnitude random key (|c| < 2^19) pins FP64 on key values with every bit position in use.
"""
import ctypes
import os

import numpy as np
import pytest

import tfhe_b200 as tb
from tfhe_oracle import torus_diff

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")
FORMS = [tb.FP64, tb.SPLIT_FP32]


def pdict(p):
    return dict(n=p.n, N=p.N, k=p.k, l=p.l, Bgbit=p.Bgbit, ks_t=p.ks_t, ks_basebit=p.ks_basebit)


def gpu_woks(ck, p, x, mu, precision):
    x = np.ascontiguousarray(x, dtype=np.int32)
    out = torch.full((len(x), p.k * p.N + 1), -7, dtype=torch.int32, device="cuda")
    ck.bootstrap_woks_device(torch.from_numpy(x).cuda(), out, len(x), int(mu), precision=precision)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.fixture(scope="module")
def rings():
    out = {}
    for name, p, seed in (("default", tb.default_params(), 91), ("large", tb.large_params(), 92)):
        sk, ck = tb.keygen(p, seed=seed)
        ck.to_device(0)
        bsk, ksk = ck.export()
        out[name] = (p, ck, bsk)
    return out


def golden_rows(rows, n):
    """Input ciphertexts whose a_i and b are the reference's mod-switch golden phases."""
    g = np.load(os.path.join(GOLDEN, "numerics.npz"))
    ph = g["phases"].astype(np.int32)
    need = rows * (n + 1)
    reps = -(-need // len(ph))
    return np.tile(ph, reps)[:need].reshape(rows, n + 1)


@pytest.mark.parametrize("precision", FORMS)
@pytest.mark.parametrize("ring", ["default", "large"])
def test_zero_rotation_bootstrap_bit_exact(oracle, rings, ring, precision):
    p, ck, bsk = rings[ring]
    rng = np.random.default_rng(5 + p.N + precision)
    b = np.array([0, 1, -1, 2**31 - 1, -2**31, 2**29, -2**29, 2**20 + 3] +
                 list(rng.integers(-2**31, 2**31, 24)), dtype=np.int64).astype(np.int32)
    x = np.zeros((len(b), p.n + 1), np.int32)
    x[:, p.n] = b
    for mu in (oracle.modswitch_to(1, 8), oracle.modswitch_to(-3, 16), 123456789):
        got = gpu_woks(ck, p, x, mu, precision)
        want = oracle.bootstrap_woks(pdict(p), bsk, mu, x)
        assert (got == want).all(), f"N={p.N} mu={mu}: {(got != want).sum()} words differ"


def coarse_key(p, shift, seed):
    rng = np.random.default_rng(seed)
    h = rng.integers(-2, 2, (p.n, (p.k + 1) * p.l, p.k + 1, p.N))
    return (h * (1 << shift)).astype(np.int32)


@pytest.mark.parametrize("N", [1024, 2048])
def test_coarse_key_bootstrap_bit_exact_both_forms(oracle, N):
    # N = 1024: the default parameters (n = 630, all 630 steps); N = 2048: the larger ring's l and
    # Bgbit with n = 48 steps so that the oracle's exact products finish in seconds
    p = tb.default_params() if N == 1024 else tb.make_params(48, 2048, 1, 3, 8, 8, 2)
    shift = tb.api.lib().tfheb_default_split_shift(ctypes.byref(p))
    bsk = coarse_key(p, shift, seed=N)
    ksk = np.zeros((p.k * p.N, p.ks_t, 1 << p.ks_basebit, p.n + 1), np.int32)  # unused: no keyswitch
    ck = tb.CloudKey.from_raw(p, bsk, ksk).to_device(0)
    g = np.load(os.path.join(GOLDEN, "numerics.npz"))
    msizes = list(g["msizes"])
    col = msizes.index(2 * p.N)
    # the oracle's mod-switch is the reference's on these phases
    sample = np.arange(0, len(g["phases"]), 67)
    assert all(oracle.modswitch_from(int(g["phases"][i]), 2 * p.N) == int(g["ms_from"][col][i]) for i in sample)
    rows = 3 if N == 1024 else 4
    x = golden_rows(rows, p.n)
    # mu = 1/8 gives digits that are powers of two; with 2^26-granular keys (N = 2048) every product
    # then wraps to zero, so a mu with mixed bits is used as well
    mus = [oracle.modswitch_to(1, 8), 0x12345679] if N == 1024 else [0x12345679]
    for mu in mus:
        want = oracle.bootstrap_woks(pdict(p), bsk, mu, x)
        assert np.count_nonzero(want[:, :p.k * p.N]) > 0, "the masks must be non-zero for the pin to mean much"
        for precision in FORMS:
            got = gpu_woks(ck, p, x, mu, precision)
            d = torus_diff(got, want)
            assert (got == want).all(), (f"N={N} mu={mu:#x} precision {precision}: {np.count_nonzero(d)} words "
                                         f"differ, max |diff| {np.abs(d).max()}")


def test_small_key_bootstrap_bit_exact_fp64(oracle):
    # every key coefficient in [-2^19, 2^19): products below 2^38, exact in FP64 for all 630 steps
    p = tb.default_params()
    rng = np.random.default_rng(19)
    bsk = rng.integers(-2**19, 2**19, (p.n, (p.k + 1) * p.l, p.k + 1, p.N)).astype(np.int32)
    ksk = np.zeros((p.k * p.N, p.ks_t, 1 << p.ks_basebit, p.n + 1), np.int32)
    ck = tb.CloudKey.from_raw(p, bsk, ksk).to_device(0, precisions=(tb.FP64,))
    x = np.concatenate([golden_rows(1, p.n), rng.integers(-2**31, 2**31, (1, p.n + 1)).astype(np.int32)])
    mu = oracle.modswitch_to(1, 8)
    got = gpu_woks(ck, p, x, mu, tb.FP64)
    want = oracle.bootstrap_woks(pdict(p), bsk, mu, x)
    assert (got == want).all(), f"{(got != want).sum()} words differ"
