"""The allocation-free gate entry point (tfheb_gate_batch_device_noalloc) against the regular one.

Callers that cannot allocate device memory -- real-time or signal-handling paths that must not
enter the allocator, processes whose device memory belongs to a framework's pool -- use the variant
whose scratch lives in a fixed device array inside the library.
It launches the same kernels, so on the same inputs its ciphertexts must equal the regular entry
point's bit for bit (the kernels are deterministic); two calls in a row check that the shared
array's leftover contents from the previous call do not leak into the next one.
"""
import ctypes

import numpy as np
import pytest

import tfhe_b200 as tb

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

V = ctypes.c_void_p


def noalloc(ck, gate, precision, count, a, b, c, out, stream=None):
    L = tb.api.lib()
    L.tfheb_gate_batch_device_noalloc.argtypes = [V, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, V, V, V, V, V]
    ptr = lambda t: None if t is None else V(t.data_ptr())  # noqa: E731
    return L.tfheb_gate_batch_device_noalloc(ck.h, gate, precision, count, ptr(a), ptr(b), ptr(c), ptr(out), stream)


@pytest.fixture(scope="module")
def keys():
    p = tb.default_params()
    sk, ck = tb.keygen(p, seed=314)
    ck.to_device(0)
    return p, sk, ck


@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_noalloc_matches_regular_entry_point_on_two_calls(keys, precision):
    p, sk, ck = keys
    rng = np.random.default_rng(27 + precision)
    calls = [(tb.api.NAND, 300), (tb.api.MUX, 120)]  # second call: different gate, shorter batch
    for gate, count in calls:
        bits = rng.integers(0, 2, (3, count))
        a, b, c = (torch.from_numpy(sk.encrypt(bits[i], seed=40 + i)).cuda() for i in range(3))
        cc = c if gate == tb.api.MUX else None
        want = torch.zeros_like(a)
        got = torch.full_like(a, -1)
        ck.gate_device(gate, a, b, cc, want, count, precision=precision)
        ck.synchronize()
        assert noalloc(ck, gate, precision, count, a, b, cc, got) == 0, tb.api.lib().tfheb_last_error()
        ck.synchronize()
        torch.cuda.synchronize()
        assert torch.equal(got, want), f"gate {gate}: no-alloc output differs from the regular entry point"
        dec, _ = sk.decrypt(got.cpu().numpy())
        truth = 1 - (bits[0] & bits[1]) if gate == tb.api.NAND else np.where(bits[0] == 1, bits[1], bits[2])
        assert (dec == truth).all()


def test_noalloc_rejects_batches_beyond_its_fixed_scratch(keys):
    p, sk, ck = keys
    count = 4096  # ~60 MB of scratch at the default parameters, the fixed array holds 8 MiB
    a = torch.zeros((count, p.n + 1), dtype=torch.int32, device="cuda")
    out = torch.zeros_like(a)
    st = noalloc(ck, tb.api.NAND, tb.FP64, count, a, a, None, out)
    assert st == 1  # TFHEB_ERR_INVALID
    assert b"scratch" in tb.api.lib().tfheb_last_error()


def test_noalloc_checks_buffers_and_counts_like_the_regular_entry_point(keys):
    p, sk, ck = keys
    L = tb.api.lib()
    # an empty batch needs no buffers
    assert noalloc(ck, tb.api.NAND, tb.FP64, 0, None, None, None, None) == 0
    # a host buffer is refused on the host, before any kernel could touch it
    host = np.zeros((4, p.n + 1), np.int32)
    d = torch.zeros((4, p.n + 1), dtype=torch.int32, device="cuda")
    L.tfheb_gate_batch_device_noalloc.argtypes = [V, ctypes.c_int32, ctypes.c_int32, ctypes.c_int32, V, V, V, V, V]
    st = L.tfheb_gate_batch_device_noalloc(ck.h, tb.api.NAND, tb.FP64, 4, V(host.ctypes.data), V(d.data_ptr()),
                                           None, V(d.data_ptr()), None)
    assert st == 1 and b"d_a" in L.tfheb_last_error()
    # NOT is one negation kernel, counted like the regular entry point counts it
    bits = np.array([0, 1, 1, 0])
    a = torch.from_numpy(sk.encrypt(bits, seed=9)).cuda()
    out = torch.zeros_like(a)
    before = tb.kernel_launches()
    assert noalloc(ck, tb.api.NOT, tb.FP64, 4, a, None, None, out) == 0
    torch.cuda.synchronize()
    assert tb.kernel_launches() - before == 1
    assert (sk.decrypt(out.cpu().numpy())[0] == 1 - bits).all()
