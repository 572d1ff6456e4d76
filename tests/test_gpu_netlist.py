"""Levelled netlist evaluation (a seeded random layered circuit in the shape of the long-run and
addition programs of the reference's test suite) against the plaintext evaluation of the same
circuit, eagerly and through the captured CUDA graph; and one batch of mixed gate types over wire
rows (tfheb_gate_batch_mixed_device) against per-type batches."""
import numpy as np
import pytest

import tfhe_b200 as tb
from tfhe_b200.api import Netlist, eval_plain, random_netlist

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

ALL_GATES = {c: 1.0 for c in range(13)}


@pytest.fixture(scope="module")
def keys():
    p = tb.default_params()
    sk, ck = tb.keygen(p, seed=808)
    ck.to_device(0)
    return p, sk, ck


@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_netlist_all_gate_types_matches_plaintext(keys, precision):
    p, sk, ck = keys
    rng = np.random.default_rng(5 + precision)
    ni, gates, ia, ib, ic = random_netlist(rng, levels=8, width_lo=16, width_hi=160, mix=ALL_GATES)
    bits = rng.integers(0, 2, ni)
    truth = eval_plain(ni, gates, ia, ib, ic, bits)
    nl = Netlist(ck, ni, gates, ia, ib, ic)
    levels, width = nl.info()
    # the level count is the critical path length; gates with slack may move to fill waves, so a
    # level can be wider than any layer of the generated circuit
    depth = np.zeros(ni + len(gates), np.int64)
    for g, code in enumerate(gates):
        srcs = (ia[g],) if code >= tb.api.NOT else ((ia[g], ib[g], ic[g]) if code == tb.api.MUX else (ia[g], ib[g]))
        depth[ni + g] = 1 + max(depth[s] for s in srcs)
    assert levels == depth.max() and width <= len(gates)
    wires = torch.zeros((ni + len(gates), p.n + 1), dtype=torch.int32, device="cuda")
    wires[:ni] = torch.from_numpy(sk.encrypt(bits, seed=9))
    nl.run(wires, precision=precision, use_graph=False)
    ck.synchronize()
    got, _ = sk.decrypt(wires.cpu().numpy())
    assert (got == truth).all(), f"{int((got != truth).sum())} wrong wires (eager)"
    # graph: the first graph run evaluates eagerly and captures, the second replays the graph
    for _ in range(2):
        wires[ni:] = 0
        nl.run(wires, precision=precision, use_graph=True)
        ck.synchronize()
        got, _ = sk.decrypt(wires.cpu().numpy())
        assert (got == truth).all(), f"{int((got != truth).sum())} wrong wires (graph)"
    nl.free()


def test_netlist_rejects_forward_references(keys):
    p, sk, ck = keys
    with pytest.raises(tb.api.TfhebError):
        Netlist(ck, 2, np.array([0]), np.array([0]), np.array([2]))  # gate 0 reads its own output wire


@pytest.mark.parametrize("precision", [tb.FP64, tb.SPLIT_FP32])
def test_mixed_batch_matches_per_type_batches(keys, precision):
    p, sk, ck = keys
    rng = np.random.default_rng(70 + precision)
    W, count = 300, 220
    bits = rng.integers(0, 2, W)
    wires0 = sk.encrypt(bits, seed=12)
    codes = rng.integers(0, 13, count).astype(np.int32)
    ia, ib, ic = (rng.integers(0, W, count).astype(np.int32) for _ in range(3))
    out = rng.permutation(W)[:count].astype(np.int32)  # distinct rows, many of them operands too
    d = torch.from_numpy(wires0.copy()).cuda()
    ck.gate_mixed_device(codes, ia, ib, ic, out, d, W, precision=precision)
    ck.synchronize()
    got = d.cpu().numpy()
    want = wires0.copy()
    for code in range(13):
        sel = np.nonzero(codes == code)[0]
        if len(sel) == 0:
            continue
        if code == tb.api.NOT:
            res = (-wires0[ia[sel]].astype(np.int64)).astype(np.int32)
        elif code == tb.api.COPY:
            res = wires0[ia[sel]]
        else:
            res = ck.gate(code, wires0[ia[sel]], wires0[ib[sel]], wires0[ic[sel]] if code == tb.api.MUX else None,
                          precision=precision)
        want[out[sel]] = res
    assert (got == want).all()
    dec, _ = sk.decrypt(got[out])
    a, b, c = bits[ia], bits[ib], bits[ic]
    truth = {0: 1 - (a & b), 1: a | b, 2: a & b, 3: a ^ b, 4: 1 - (a ^ b), 5: 1 - (a | b), 6: (1 - a) & b,
             7: a & (1 - b), 8: (1 - a) | b, 9: a | (1 - b), 10: np.where(a == 1, b, c), 11: 1 - a, 12: a}
    expect = np.choose(codes, [truth[k] for k in range(13)])
    assert (dec == expect).all()


def test_mixed_batch_rejects_bad_rows(keys):
    p, sk, ck = keys
    d = torch.zeros((4, p.n + 1), dtype=torch.int32, device="cuda")
    g = np.array([0, 0], np.int32)
    with pytest.raises(tb.api.TfhebError, match="operand row out of range"):
        ck.gate_mixed_device(g, [0, 1], [2, 4], None, [2, 3], d, 4)
    with pytest.raises(tb.api.TfhebError, match="output row written twice"):
        ck.gate_mixed_device(g, [0, 1], [2, 3], None, [3, 3], d, 4)
    with pytest.raises(tb.api.TfhebError, match="output row out of range"):
        ck.gate_mixed_device(g, [0, 1], [2, 3], None, [0, -1], d, 4)
