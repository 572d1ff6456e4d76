"""Generate the golden vectors under tests/golden/ by running the reference library itself.

The reference (tfhe v1.1, spqlios-fma backend) ships no golden vectors or fixtures, so these are
produced here from fixed seeds by the reference build in oracle/_ref/ (oracle/ref.mk) through the
thin ctypes shim oracle/ref_shim.cpp.  Run from the repository root after building the reference:

    make -f oracle/ref.mk REF=<path to the tfhe checkout>
    python tests/golden/make_golden.py

Every fixture is a small .npz; the tests that read them never need the reference at run time.
"""
import ctypes
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "tests"))

from tfhe_ref import RefLib  # noqa: E402


def numerics(ref, rng):
    phases = np.concatenate([
        rng.integers(-2**31, 2**31, 2000, dtype=np.int64),
        np.array([0, 1, -1, 2**31 - 1, -2**31, 2**20, -2**20, 2**21 - 1, 2**21, 2**21 + 1], np.int64),
    ]).astype(np.int32)
    msizes = np.array([4, 8, 16, 1024, 2048, 4096], np.int32)
    ms_from = np.array([[ref.modswitch_from(int(p), int(m)) for p in phases] for m in msizes], np.int32)
    mus = np.arange(-10, 11, dtype=np.int32)
    ms_to = np.array([[ref.modswitch_to(int(u), int(m)) for u in mus] for m in msizes], np.int32)
    np.savez_compressed(os.path.join(HERE, "numerics.npz"), phases=phases, msizes=msizes,
                        ms_from=ms_from, mus=mus, ms_to=ms_to)


def decomposition(ref, rng):
    out = {}
    for (N, l, bgbit) in [(1024, 3, 7), (2048, 3, 8), (1024, 2, 10)]:
        polys = rng.integers(-2**31, 2**31, (3, N), dtype=np.int64).astype(np.int32)
        polys[2, :8] = [0, 1, -1, 2**31 - 1, -2**31, 1 << (31 - l * bgbit), -(1 << (31 - l * bgbit)), 12345]
        digits = np.stack([ref.decompose(N, l, bgbit, p) for p in polys])
        tag = f"N{N}_l{l}_b{bgbit}"
        out[f"{tag}_polys"] = polys
        out[f"{tag}_digits"] = digits
    np.savez_compressed(os.path.join(HERE, "decomposition.npz"), **out)


def rotations(ref, rng):
    out = {}
    for N in (1024, 2048):
        poly = rng.integers(-2**31, 2**31, N, dtype=np.int64).astype(np.int32)
        avals = np.array([0, 1, 7, N // 2, N - 1, N, N + 1, N + N // 3, 2 * N - 1], np.int32)
        out[f"N{N}_poly"] = poly
        out[f"N{N}_a"] = avals
        out[f"N{N}_xai"] = np.stack([ref.rotate(N, int(a), False, poly) for a in avals])
        out[f"N{N}_xai_minus_one"] = np.stack([ref.rotate(N, int(a), True, poly) for a in avals])
    np.savez_compressed(os.path.join(HERE, "rotations.npz"), **out)


def extraction(ref, rng):
    out = {}
    for (N, k) in [(1024, 1), (2048, 1), (512, 2)]:
        tlwe = rng.integers(-2**31, 2**31, ((k + 1), N), dtype=np.int64).astype(np.int32)
        out[f"N{N}_k{k}_tlwe"] = tlwe
        out[f"N{N}_k{k}_lwe"] = ref.extract(N, k, tlwe)
    np.savez_compressed(os.path.join(HERE, "extraction.npz"), **out)


def products(ref, rng):
    out = {}
    for N in (512, 1024, 2048):
        ip = rng.integers(-64, 64, (2, N), dtype=np.int64).astype(np.int32)
        tp = rng.integers(-2**31, 2**31, (2, N), dtype=np.int64).astype(np.int32)
        out[f"N{N}_int"] = ip
        out[f"N{N}_torus"] = tp
        out[f"N{N}_naive"] = np.stack([ref.poly_mult(2, N, ip[i], tp[i]) for i in range(2)])
        out[f"N{N}_karatsuba"] = np.stack([ref.poly_mult(1, N, ip[i], tp[i]) for i in range(2)])
        if N == 1024:
            out[f"N{N}_fft"] = np.stack([ref.poly_mult(0, N, ip[i], tp[i]) for i in range(2)])
    np.savez_compressed(os.path.join(HERE, "products.npz"), **out)


def gates_small(ref, rng):
    # N=1024 (the only ring degree the reference's FFT supports: its key generation corrupts
    # memory at any other N) with a tiny LWE dimension so the keys fit in a fixture.  Gate outputs are stored with their decrypted bits and phases.
    p = dict(n=16, N=1024, k=1, l=3, Bgbit=7, ks_t=8, ks_basebit=2)
    keys = ref.keygen(custom=p, ks_stdev=2**-15, bk_stdev=2**-25, seed=77)
    lwe_key, tlwe_key, ksk, bsk = keys.export()
    G = 8
    bits = rng.integers(0, 2, (3, 13 * G)).astype(np.int32)
    ca, cb, cc = (keys.encrypt(bits[i]) for i in range(3))
    gate_codes = np.repeat(np.arange(13, dtype=np.int32), G)
    outs = np.zeros_like(ca)
    for code in range(13):
        sl = slice(code * G, (code + 1) * G)
        outs[sl] = keys.gate(code, ca[sl], cb[sl], cc[sl] if code == 10 else None)
    out_bits, out_phase = keys.decrypt(outs)
    # lweKeySwitch on random dimension-N inputs (plus all-zero and all-ones edge rows)
    ks_in = rng.integers(-2**31, 2**31, (24, p["k"] * p["N"] + 1), dtype=np.int64).astype(np.int32)
    ks_in[0, :] = 0
    ks_in[1, :] = -1
    ks_out = keys.keyswitch(ks_in)
    np.savez_compressed(os.path.join(HERE, "gates_small.npz"), params=np.array(list(p.values()), np.int32),
                        lwe_key=lwe_key, tlwe_key=tlwe_key, ksk=ksk, bsk=bsk,
                        bits=bits, ca=ca, cb=cb, cc=cc, gate_codes=gate_codes,
                        outputs=outs, out_bits=out_bits, out_phase=out_phase,
                        ks_inputs=ks_in, ks_outputs=ks_out)
    keys.free()


def noise_default(ref, rng):
    # Output-noise statistics of the reference's bootsNAND at the default 128-bit parameters:
    # phase error = phase - (+-1/8) in Torus32 units, over M gates (8 host threads).
    keys = ref.keygen(custom=None, seed=99)
    M = 8000
    bits = rng.integers(0, 2, (2, M)).astype(np.int32)
    ca, cb = keys.encrypt(bits[0]), keys.encrypt(bits[1])
    outs = np.zeros_like(ca)
    threads = 8
    keys.bench_gates(0, threads, M // threads, ca, cb, None, outs)
    got, phase = keys.decrypt(outs)
    truth = 1 - (bits[0] & bits[1])
    mu = np.where(truth == 1, 1 << 29, -(1 << 29)).astype(np.int64)
    err = ((phase.astype(np.int64) - mu + 2**31) % 2**32) - 2**31
    np.savez_compressed(os.path.join(HERE, "noise_default.npz"), gates=np.int64(M),
                        errors=np.int64((got != truth).sum()), err_mean=err.mean(), err_var=err.var(),
                        err_max=np.abs(err).max())
    keys.free()


def keyswitch_general(ref, rng):
    # lweKeySwitch with a keyswitch shape other than the default's t=8, basebit=2 (t=4, basebit=3:
    # 8 rows per digit position, a 12-bit decomposition), which only the general per-sample kernel
    # serves.  N=1024 as above; n=8 keeps the keyswitching key at 1.2 MB.  Own generator, so that it
    # can be regenerated alone.
    rng = np.random.default_rng(20261203)
    p = dict(n=8, N=1024, k=1, l=3, Bgbit=7, ks_t=4, ks_basebit=3)
    keys = ref.keygen(custom=p, ks_stdev=2**-15, bk_stdev=2**-25, seed=78)
    _, _, ksk, _ = keys.export(bsk=False)
    ks_in = rng.integers(-2**31, 2**31, (40, p["k"] * p["N"] + 1), dtype=np.int64).astype(np.int32)
    ks_in[0, :] = 0
    ks_in[1, :] = -1
    ks_out = keys.keyswitch(ks_in)
    np.savez_compressed(os.path.join(HERE, "keyswitch_t4b3.npz"), params=np.array(list(p.values()), np.int32),
                        ksk=ksk, ks_inputs=ks_in, ks_outputs=ks_out)
    keys.free()


GENERATORS = [numerics, decomposition, rotations, extraction, products, gates_small, noise_default,
              keyswitch_general]


def main(names):
    """Writes every fixture, or only those whose generator is named on the command line."""
    ref = RefLib.load(required=True)
    rng = np.random.default_rng(20240601)
    for gen in GENERATORS:
        if not names or gen.__name__ in names:
            gen(ref, rng)
    print("golden vectors written to", HERE)


if __name__ == "__main__":
    main(sys.argv[1:])
