"""Edge cases of the entry points on the GPU: empty batches everywhere, bootstrap-free gates, a
netlist without gates, and one batch far above a wave (the largest single call the bench makes is
4096 gates; this one is 20,000)."""
import numpy as np
import pytest

import tfhe_b200 as tb
from tfhe_b200.api import Netlist, NetlistMulti

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def keys():
    p = tb.default_params()
    sk, ck = tb.keygen(p, seed=77)
    ck.to_device(0)
    return p, sk, ck


def test_empty_batches_on_every_entry_point(keys):
    p, sk, ck = keys
    n1, kn1 = p.n + 1, p.k * p.N + 1
    e = np.zeros((0, n1), np.int32)
    for code in (tb.api.NAND, tb.api.MUX, tb.api.NOT):
        out = ck.gate(code, e, e if code != tb.api.NOT else None, e if code == tb.api.MUX else None)
        assert out.shape == (0, n1)
    d = torch.zeros((1, n1), dtype=torch.int32, device="cuda")
    dk = torch.zeros((1, kn1), dtype=torch.int32, device="cuda")
    ck.gate_device(tb.api.NAND, d, d, None, d, 0)
    ck.bootstrap_woks_device(d, dk, 0, 1 << 29)
    ck.keyswitch_device(dk, d, 0)
    ck.blind_rotate_device(torch.zeros((1, 1), dtype=torch.int32, device="cuda"),
                           torch.zeros((1, 2 * p.N), dtype=torch.int32, device="cuda"), 0, 1)
    ck.gate_mixed_device([], [], [], [], [], d, 1)
    assert (tb.gate_batch_multi([ck], tb.api.NAND, e, e).shape == (0, n1))
    ck.synchronize()


@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_bootstrap_free_gates_on_host_and_device(keys, precision):
    p, sk, ck = keys
    bits = np.array([0, 1, 1, 0, 1])
    a = sk.encrypt(bits, seed=3)
    assert (ck.gate(tb.api.NOT, a, precision=precision) == (-a.astype(np.int64)).astype(np.int32)).all()
    assert (ck.gate(tb.api.COPY, a, precision=precision) == a).all()
    d, out = torch.from_numpy(a).cuda(), torch.zeros((5, p.n + 1), dtype=torch.int32, device="cuda")
    ck.gate_device(tb.api.NOT, d, None, None, out, 5, precision=precision)
    ck.synchronize()
    assert (sk.decrypt(out.cpu().numpy())[0] == 1 - bits).all()


def test_netlist_without_gates(keys):
    p, sk, ck = keys
    inputs = sk.encrypt(np.array([1, 0, 1]), seed=4)
    nl = Netlist(ck, 3, np.zeros(0, np.int32), np.zeros(0, np.int32))
    assert nl.info() == (0, 0)
    w = torch.from_numpy(inputs.copy()).cuda()
    nl.run(w, use_graph=False)
    nl.run(w, use_graph=True)
    ck.synchronize()
    assert (w.cpu().numpy() == inputs).all()
    got = NetlistMulti([ck], 3, np.zeros(0, np.int32), np.zeros(0, np.int32)).run(inputs)
    assert (got == inputs).all()


def test_one_call_of_twenty_thousand_gates(keys):
    p, sk, ck = keys
    rng = np.random.default_rng(5)
    x, y = rng.integers(0, 2, 20000), rng.integers(0, 2, 20000)
    out = ck.gate(tb.api.AND, sk.encrypt(x, seed=6), sk.encrypt(y, seed=7), precision=tb.SPLIT_FP32)
    got, _ = sk.decrypt(out)
    assert (got == (x & y)).all()
