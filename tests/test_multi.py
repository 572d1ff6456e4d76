"""Replica sharding of one batch across several cloud keys (tfheb_gate_batch_multi).

Host-side checks run without a GPU; the GPU tests compare the sharded result with one
tfheb_gate_batch call over the whole batch, bit for bit.  With one GPU, the second key lives on
the same device: the shards are independent launches on two streams, so that is the same code
path a second GPU takes.
"""
import numpy as np
import pytest

import tfhe_b200 as tb
from tfhe_b200.api import TfhebError

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
