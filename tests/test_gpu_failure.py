"""Failure detection on the GPU without a fault: the key-streaming warp of the blind rotation, or
the copy-issuing thread of a keyswitch kernel, is told to issue nothing, so every consumer wait runs
out after a short limit; the launch must come back with TFHEB_ERR_TIMEOUT (no hang, no trap) and the
same key must compute correctly afterwards."""
import os

import numpy as np
import pytest

import tfhe_b200 as tb

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_stalled_key_stream_reports_timeout_and_context_survives(precision):
    g = np.load(os.path.join(GOLDEN, "gates_small.npz"))
    p = tb.make_params(*map(int, g["params"]))
    ck = tb.CloudKey.from_raw(p, g["bsk"], g["ksk"]).to_device(0)
    sk = tb.SecretKey.from_raw(p, g["lwe_key"], g["tlwe_key"])
    sel = g["gate_codes"] == 0
    ck.set_wait_timeout(0.05)
    ck.test_stall_key_stream(True)
    with pytest.raises(tb.api.TfhebError) as exc:
        ck.gate(tb.api.NAND, g["ca"][sel], g["cb"][sel], precision=precision)
    assert exc.value.status == tb.api.TIMEOUT
    ck.test_stall_key_stream(False)
    ck.set_wait_timeout(1.0)
    out = ck.gate(tb.api.NAND, g["ca"][sel], g["cb"][sel], precision=precision)
    bits, _ = sk.decrypt(out)
    assert (bits == g["out_bits"][sel]).all()


# tiled, register-key, tensor-core: all stream key rows through a ring
@pytest.mark.parametrize("kernel", [2, 3, 4])
def test_stalled_keyswitch_ring_reports_timeout_and_context_survives(kernel):
    torch = pytest.importorskip("torch")
    g = np.load(os.path.join(GOLDEN, "gates_small.npz"))
    p = tb.make_params(*map(int, g["params"]))
    ck = tb.CloudKey.from_raw(p, g["bsk"], g["ksk"]).to_device(0)
    x = torch.from_numpy(np.ascontiguousarray(g["ks_inputs"], dtype=np.int32)).cuda()
    out = torch.zeros((len(x), p.n + 1), dtype=torch.int32, device="cuda")
    ck.set_keyswitch_kernel(kernel)
    ck.set_wait_timeout(0.05)
    ck.test_stall_key_stream(True)
    with pytest.raises(tb.api.TfhebError) as exc:
        ck.keyswitch_device(x, out, len(x))
        ck.synchronize()
    assert exc.value.status == tb.api.TIMEOUT
    ck.test_stall_key_stream(False)
    ck.set_wait_timeout(1.0)
    ck.keyswitch_device(x, out, len(x))
    ck.synchronize()
    assert (out.cpu().numpy() == g["ks_outputs"]).all()
