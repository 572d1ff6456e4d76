"""tfheb_gate_batch on host buffers against tfheb_gate_batch_device on the same inputs, bit for bit
and decrypting to the truth table, for batches of several blind-rotation waves, a batch one gate
above a wave, MUX, and a bootstrap-free gate; and the descriptor cache across calls of different
sizes and gates."""
import numpy as np
import pytest

import tfhe_b200 as tb

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

TRUTH = {tb.api.NAND: lambda a, b, c: 1 - (a & b), tb.api.XOR: lambda a, b, c: a ^ b,
         tb.api.MUX: lambda a, b, c: np.where(a == 1, b, c), tb.api.NOT: lambda a, b, c: 1 - a}


@pytest.fixture(scope="module")
def keys():
    p = tb.default_params()
    sk, ck = tb.keygen(p, seed=2024)
    ck.to_device(0)
    return p, sk, ck


# 2500 NAND: several waves; 1500 MUX: 3000 bootstraps; 1037 XOR: one gate above a split-FP32 wave of
# 148 x 7; 3000 NOT: no bootstrap
@pytest.mark.parametrize("gate,count", [(tb.api.NAND, 2500), (tb.api.MUX, 1500), (tb.api.XOR, 1037),
                                        (tb.api.NOT, 3000)])
@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_chunked_host_batch_equals_device_batch(keys, gate, count, precision):
    p, sk, ck = keys
    rng = np.random.default_rng(gate * 10 + precision)
    bits = [rng.integers(0, 2, count) for _ in range(3)]
    cts = [sk.encrypt(x, seed=30 + i) for i, x in enumerate(bits)]
    binary = gate != tb.api.NOT
    mux = gate == tb.api.MUX
    host = ck.gate(gate, cts[0], cts[1] if binary else None, cts[2] if mux else None, precision=precision)
    d = [torch.from_numpy(x).cuda() for x in cts]
    d_out = torch.zeros_like(d[0])
    ck.gate_device(gate, d[0], d[1] if binary else None, d[2] if mux else None, d_out, count, precision=precision)
    ck.synchronize()
    assert (host == d_out.cpu().numpy()).all()
    got, _ = sk.decrypt(host)
    assert (got == TRUTH[gate](*bits)).all()


def test_descriptor_cache_across_sizes_and_gates(keys):
    # descriptors built for a larger count serve a smaller one of the same gate (a prefix); another
    # gate or a larger count rebuilds them
    p, sk, ck = keys
    rng = np.random.default_rng(3)
    x, y, z = (rng.integers(0, 2, 600) for _ in range(3))
    a, b, c = (sk.encrypt(v, seed=i) for i, v in enumerate((x, y, z)))
    for gate, n in ((tb.api.NAND, 600), (tb.api.NAND, 37), (tb.api.MUX, 300), (tb.api.NAND, 599),
                    (tb.api.MUX, 600)):
        out = ck.gate(gate, a[:n], b[:n], c[:n] if gate == tb.api.MUX else None, precision=tb.SPLIT_FP32)
        got, _ = sk.decrypt(out)
        assert (got == TRUTH[gate](x[:n], y[:n], z[:n])).all(), (gate, n)


def test_device_entry_points_reject_host_memory(keys):
    # a host array given where device memory is expected is refused before any kernel runs
    p, sk, ck = keys
    a = sk.encrypt(np.array([1, 0, 1]), seed=1)
    d = torch.from_numpy(a).cuda()
    d_out = torch.zeros_like(d)
    with pytest.raises(tb.api.TfhebError, match="d_b: not device memory"):
        ck.gate_device(tb.api.NAND, d, a, None, d_out, 3)
    with pytest.raises(tb.api.TfhebError, match="d_out: not device memory"):
        ck.gate_device(tb.api.NAND, d, d, None, np.zeros_like(a), 3)
    # the key is still usable afterwards
    ck.gate_device(tb.api.NAND, d, d, None, d_out, 3)
    ck.synchronize()
    got, _ = sk.decrypt(d_out.cpu().numpy())
    assert (got == [0, 1, 0]).all()


def test_calls_on_two_streams_use_the_key_scratch_in_order(keys):
    # two batches on one key, issued back to back on two streams with no host synchronisation: the
    # second waits on the device for the first to finish with the key's scratch
    import ctypes
    p, sk, ck = keys
    rng = np.random.default_rng(11)
    n = 1500
    bits = [rng.integers(0, 2, n) for _ in range(4)]
    cts = [torch.from_numpy(sk.encrypt(x, seed=50 + i)).cuda() for i, x in enumerate(bits)]
    o1, o2 = torch.zeros_like(cts[0]), torch.zeros_like(cts[0])
    s1, s2 = torch.cuda.Stream(), torch.cuda.Stream()
    torch.cuda.synchronize()
    ck.gate_device(tb.api.NAND, cts[0], cts[1], None, o1, n, precision=tb.SPLIT_FP32,
                   stream=ctypes.c_void_p(s1.cuda_stream))
    ck.gate_device(tb.api.XOR, cts[2], cts[3], None, o2, n, precision=tb.SPLIT_FP32,
                   stream=ctypes.c_void_p(s2.cuda_stream))
    torch.cuda.synchronize()
    g1, _ = sk.decrypt(o1.cpu().numpy())
    g2, _ = sk.decrypt(o2.cpu().numpy())
    assert (g1 == 1 - (bits[0] & bits[1])).all()
    assert (g2 == (bits[2] ^ bits[3])).all()
    # and bit for bit what one stream gives
    r1 = torch.zeros_like(o1)
    ck.gate_device(tb.api.NAND, cts[0], cts[1], None, r1, n, precision=tb.SPLIT_FP32)
    ck.synchronize()
    assert torch.equal(r1, o1)


@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_small_batches_match_large_batches_bit_for_bit(keys, precision):
    # 20 gates fit one wave with one bootstrap per CTA, so they run on a small-batch variant (or, after
    # the autotuner, on whatever it measured fastest); 300 / 592 / 740 / 888 gates need 3 / 4 / 5 / 6
    # bootstraps per CTA (148 SMs), the small-batch variants with that many teams; 2000 gates run on
    # the tuned variant
    p, sk, ck = keys
    rng = np.random.default_rng(90 + precision)
    x, y = rng.integers(0, 2, 2000), rng.integers(0, 2, 2000)
    a, b = sk.encrypt(x, seed=91), sk.encrypt(y, seed=92)
    for tuned in (False, True):
        if tuned:
            ck.autotune(precision, boots=2000)
        big = ck.gate(tb.api.NAND, a, b, precision=precision)
        for n_ in (20, 300, 592, 740, 888):
            part = ck.gate(tb.api.NAND, a[:n_], b[:n_], precision=precision)
            assert (part == big[:n_]).all(), f"{n_} gates differ from the large batch"
        got, _ = sk.decrypt(big)
        assert (got == 1 - (x & y)).all()


@pytest.fixture(scope="module")
def large_keys():
    p = tb.large_params()
    sk, ck = tb.keygen(p, seed=2048)
    ck.to_device(0)
    return p, sk, ck


@pytest.mark.parametrize("ring", ["default", "large"])
@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_every_tuned_variant_gives_the_same_bits(request, ring, precision):
    # 1036 gates need 7 bootstraps per CTA for one wave, no fewer than any candidate packs, so no
    # small-batch variant stands in: packing, ring depth, paired transforms and who streams the key
    # must not change a bit
    p, sk, ck = request.getfixturevalue("keys" if ring == "default" else "large_keys")
    rng = np.random.default_rng(120 + precision)
    x, y = rng.integers(0, 2, 1036), rng.integers(0, 2, 1036)
    a, b = sk.encrypt(x, seed=121), sk.encrypt(y, seed=122)
    G, _ = ck.br_variants(precision)
    outs = []
    try:
        for v in range(len(G)):
            ck.set_br_variant(precision, v)
            outs.append(ck.gate(tb.api.NAND, a, b, precision=precision))
    finally:
        ck.set_br_variant(precision, 0)
    for o in outs[1:]:
        assert (o == outs[0]).all()
    got, _ = sk.decrypt(outs[0])
    assert (got == 1 - (x & y)).all()
