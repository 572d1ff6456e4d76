"""GPU engine driven by keys made by the reference library itself (oracle/_ref, built from the
reference's sources): the reference generates keys and ciphertexts at the default 128-bit
parameters, the engine imports the raw keys and evaluates gates on the GPU, and the reference
decrypts the results.  Also: the GPU keyswitch equals the reference's lweKeySwitch bit for bit on
the reference's own keyswitching key.  Skipped when the reference build did not travel with the
checkout."""
import numpy as np
import pytest

import tfhe_b200 as tb
from tfhe_ref import RefLib

torch = pytest.importorskip("torch")
pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not RefLib.available(), reason="reference build (oracle/_ref) not present")]

TRUTH = {0: lambda a, b, c: 1 - (a & b), 3: lambda a, b, c: a ^ b, 10: lambda a, b, c: np.where(a == 1, b, c)}


@pytest.fixture(scope="module")
def ref_keys():
    ref = RefLib.load()
    keys = ref.keygen(custom=None, seed=1234)
    p = tb.default_params()
    lk, tk, ksk, bsk = keys.export()
    ck = tb.CloudKey.from_raw(p, bsk, ksk).to_device(0)
    yield keys, p, ck, ksk
    keys.free()


@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_reference_keys_gates_decrypt_with_reference(ref_keys, precision):
    keys, p, ck, _ = ref_keys
    rng = np.random.default_rng(77 + precision)
    G = 256
    a, b, c = rng.integers(0, 2, (3, G)).astype(np.int32)
    ca, cb, cc = keys.encrypt(a), keys.encrypt(b), keys.encrypt(c)
    for code, fn in TRUTH.items():
        out = ck.gate(code, ca, cb, cc if code == 10 else None, precision=precision)
        bits, _ = keys.decrypt(out)
        assert (bits == fn(a, b, c)).all(), f"gate {code}"
    # the reference's own gates on a few of the same inputs agree
    ref_out = keys.gate(0, ca[:8], cb[:8])
    assert (keys.decrypt(ref_out)[0] == 1 - (a[:8] & b[:8])).all()


# 32 samples run the tiled kernel; from 256 on, the default is the register-key kernel, the one the
# 4096-gate batches use
@pytest.mark.parametrize("count", [32, 256, 4096])
def test_gpu_keyswitch_equals_reference_lweKeySwitch(ref_keys, count):
    keys, p, ck, _ = ref_keys
    rng = np.random.default_rng(5 + count)
    x = rng.integers(-2**31, 2**31, (count, p.k * p.N + 1), dtype=np.int64).astype(np.int32)
    x[0] = 0
    x[-1] = -1
    out = torch.zeros((count, p.n + 1), dtype=torch.int32, device="cuda")
    ck.keyswitch_device(torch.from_numpy(x).cuda(), out, count)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    want = keys.keyswitch(x)
    assert (got == want).all(), f"{(got != want).any(axis=1).sum()} of {count} samples differ"
