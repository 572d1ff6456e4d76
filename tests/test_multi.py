"""Replica sharding across several cloud keys: one batch (tfheb_gate_batch_multi) and the levels of
a netlist (tfheb_netlist_multi_*).

Host-side checks run without a GPU; the GPU tests compare the sharded result with one
tfheb_gate_batch call over the whole batch, or one single-key netlist run, bit for bit.  With one
GPU, the other keys live on the same device: the shards are launches on their keys' own streams and
the per-level all-gather is a peer copy within the device, the same code path a second GPU takes.
"""
import numpy as np
import pytest

import tfhe_b200 as tb
from tfhe_b200.api import Netlist, NetlistMulti, TfhebError, eval_plain, random_netlist

SMALL = (100, 1024, 1, 3, 7, 8, 2)


def test_rejects_bad_arguments_without_a_gpu():
    p = tb.make_params(*SMALL)
    sk, ck = tb.keygen(p, seed=1)
    a = sk.encrypt(np.array([0, 1, 1]))
    with pytest.raises(TfhebError, match="invalid arguments"):
        tb.gate_batch_multi([], 0, a, a)
    q = tb.make_params(120, 1024, 1, 3, 7, 8, 2)
    _, other = tb.keygen(q, seed=2)
    with pytest.raises(TfhebError, match="another parameter set"):
        tb.gate_batch_multi([ck, other], 0, a, a)
    # keys that were never moved to a device: the failing shard is named
    with pytest.raises(TfhebError, match="shard 0"):
        tb.gate_batch_multi([ck, ck], 0, a, a)


def test_netlist_multi_rejects_bad_keys_without_a_gpu():
    p = tb.make_params(*SMALL)
    _, ck = tb.keygen(p, seed=1)
    _, ck2 = tb.keygen(p, seed=2)
    _, other = tb.keygen(tb.make_params(120, 1024, 1, 3, 7, 8, 2), seed=3)
    gates, ia, ib = np.array([0]), np.array([0]), np.array([1])
    with pytest.raises(TfhebError, match="repeats key 0"):
        NetlistMulti([ck, ck], 2, gates, ia, ib)
    with pytest.raises(TfhebError, match="another parameter set"):
        NetlistMulti([ck, other], 2, gates, ia, ib)
    with pytest.raises(TfhebError, match="not on a device"):
        NetlistMulti([ck, ck2], 2, gates, ia, ib)
    with pytest.raises(TfhebError, match="invalid arguments"):
        NetlistMulti([], 2, gates, ia, ib)


@pytest.fixture(scope="module")
def two_keys():
    torch = pytest.importorskip("torch")
    p = tb.default_params()
    sk, ck = tb.keygen(p, seed=31)
    bsk, ksk = ck.export()
    second = tb.CloudKey.from_raw(p, bsk, ksk)
    ck.to_device(0)
    second.to_device(1 if torch.cuda.device_count() > 1 else 0)
    return p, sk, ck, second


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_sharded_batch_equals_one_batch(two_keys, precision):
    p, sk, ck, second = two_keys
    rng = np.random.default_rng(precision)
    x, y = rng.integers(0, 2, 1001), rng.integers(0, 2, 1001)
    a, b = sk.encrypt(x, seed=5), sk.encrypt(y, seed=6)
    whole = ck.gate(0, a, b, precision=precision)
    sharded = tb.gate_batch_multi([ck, second], 0, a, b, precision=precision)
    assert (sharded == whole).all()
    bits, _ = sk.decrypt(sharded)
    assert (bits == 1 - (x & y)).all()


@pytest.mark.gpu
def test_mux_three_shards_and_empty_shards(two_keys):
    p, sk, ck, second = two_keys
    rng = np.random.default_rng(8)
    s, x, y = (rng.integers(0, 2, 257) for _ in range(3))
    cs, cx, cy = sk.encrypt(s, seed=1), sk.encrypt(x, seed=2), sk.encrypt(y, seed=3)
    out = tb.gate_batch_multi([ck, second, ck], 10, cs, cx, cy)
    assert (out == ck.gate(10, cs, cx, cy)).all()
    assert (sk.decrypt(out)[0] == np.where(s == 1, x, y)).all()
    # two gates over three keys: one shard is empty
    small = tb.gate_batch_multi([ck, second, ck], 3, cx[:2], cy[:2])
    assert (sk.decrypt(small)[0] == (x[:2] ^ y[:2])).all()


@pytest.fixture(scope="module")
def three_keys(two_keys):
    p, sk, ck, second = two_keys
    bsk, ksk = ck.export()
    third = tb.CloudKey.from_raw(p, bsk, ksk)
    third.to_device(0)
    return p, sk, ck, second, third


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
@pytest.mark.parametrize("nkeys", [2, 3])
def test_sharded_netlist_equals_one_key(three_keys, precision, nkeys):
    torch = pytest.importorskip("torch")
    p, sk, ck, second, third = three_keys
    rng = np.random.default_rng(40 + nkeys + precision)
    ni, gates, ia, ib, ic = random_netlist(rng, levels=6, width_lo=3, width_hi=200,
                                           mix={c: 1.0 for c in range(13)})
    bits = rng.integers(0, 2, ni)
    inputs = sk.encrypt(bits, seed=4)
    single = Netlist(ck, ni, gates, ia, ib, ic)
    d = torch.zeros((ni + len(gates), p.n + 1), dtype=torch.int32, device="cuda")
    d[:ni] = torch.from_numpy(inputs)
    single.run(d, precision=precision, use_graph=False)
    ck.synchronize()
    want = d.cpu().numpy()
    multi = NetlistMulti([ck, second, third][:nkeys], ni, gates, ia, ib, ic)
    got = multi.run(inputs, precision=precision)
    assert (got == want).all()
    dec, _ = sk.decrypt(got)
    assert (dec == eval_plain(ni, gates, ia, ib, ic, bits)).all()
    # a second run on the same object gives the same wires
    assert (multi.run(inputs, precision=precision) == want).all()
    multi.free()
    single.free()


@pytest.mark.gpu
def test_sharded_netlist_narrow_levels_leave_shards_empty(three_keys):
    p, sk, ck, second, third = three_keys
    # a chain: one gate per level, so two of the three shards have no bootstrapped gate on any level
    gates = np.array([0, 3, 10, 12, 7], np.int32)  # NAND, XOR, MUX, COPY, ANDYN
    ia = np.array([0, 2, 3, 4, 5])
    ib = np.array([1, 0, 1, 0, 1])
    ic = np.array([0, 0, 0, 0, 0])
    bits = np.array([1, 0])
    inputs = sk.encrypt(bits, seed=8)
    got = NetlistMulti([ck, second, third], 2, gates, ia, ib, ic).run(inputs, precision=tb.SPLIT_FP32)
    dec, _ = sk.decrypt(got)
    assert (dec == eval_plain(2, gates, ia, ib, ic, bits)).all()
