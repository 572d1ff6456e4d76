"""ctypes bindings for the C oracle (oracle/liboracle.so) -- test infrastructure only.

The oracle is the CPU restatement of the reference's gate-bootstrapping path with exact products
(oracle/oracle.h).  It is the checker for the GPU engine; the engine never calls it.
If the shared object is missing it is compiled on the spot with the system C compiler.
"""
import ctypes
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_DIR = os.path.join(ROOT, "oracle")
SO = os.path.join(ORACLE_DIR, "liboracle.so")

_V = ctypes.c_void_p


def _p(a):
    return None if a is None else a.ctypes.data_as(_V)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class OrParams(ctypes.Structure):
    _fields_ = [(f, ctypes.c_int32) for f in ("n", "N", "k", "l", "Bgbit", "ks_t", "ks_basebit")]


DEFAULT = dict(n=630, N=1024, k=1, l=3, Bgbit=7, ks_t=8, ks_basebit=2)
LARGE = dict(n=800, N=2048, k=1, l=3, Bgbit=8, ks_t=8, ks_basebit=2)


def build():
    src = os.path.join(ORACLE_DIR, "oracle.c")
    if os.path.exists(SO) and os.path.getmtime(SO) >= os.path.getmtime(src):
        return SO
    subprocess.check_call(["make", "-s", "-C", ORACLE_DIR])
    return SO


class Oracle:
    _inst = None

    def __init__(self):
        L = ctypes.CDLL(build())
        L.or_keygen.argtypes = [_V, ctypes.c_double, ctypes.c_double, ctypes.c_uint64, _V, _V, _V, _V]
        L.or_lwe_encrypt.argtypes = [ctypes.c_int32, _V, _V, ctypes.c_double, ctypes.c_uint64, ctypes.c_int32, _V]
        self.L = L

    @classmethod
    def get(cls):
        if cls._inst is None:
            cls._inst = Oracle()
        return cls._inst

    # ---- building blocks -------------------------------------------------------------------
    def modswitch_from(self, phase, msize):
        return self.L.or_modswitch_from(int(phase), int(msize))

    def modswitch_to(self, mu, msize):
        return self.L.or_modswitch_to(int(mu), int(msize))

    def decompose(self, N, l, bgbit, poly):
        out = np.zeros((l, N), np.int32)
        self.L.or_decompose(N, l, bgbit, _p(_i32(poly)), _p(out))
        return out

    def rotate(self, N, a, minus_one, poly):
        out = np.zeros(N, np.int32)
        fn = self.L.or_mul_by_xai_minus_one if minus_one else self.L.or_mul_by_xai
        fn(N, int(a), _p(_i32(poly)), _p(out))
        return out

    def extract(self, N, k, tlwe):
        out = np.zeros(k * N + 1, np.int32)
        self.L.or_extract(N, k, _p(_i32(tlwe)), _p(out))
        return out

    def negacyclic_mult(self, N, ipoly, tpoly):
        out = np.zeros(N, np.int32)
        self.L.or_negacyclic_mult(N, _p(_i32(ipoly)), _p(_i32(tpoly)), _p(out))
        return out

    def negacyclic_mult_wide(self, N, ipoly, tpoly):
        """Exact int128 product, returned as Python ints (object array)."""
        raw = np.zeros(2 * N, np.uint64)
        self.L.or_negacyclic_mult_wide(N, _p(_i32(ipoly)), _p(_i32(tpoly)), _p(raw))
        lo = raw[0::2].astype(object)
        hi = raw[1::2].astype(np.int64).astype(object)
        return np.array([int(h) * (1 << 64) + int(l_) for l_, h in zip(lo, hi)], dtype=object)

    # ---- path ------------------------------------------------------------------------------
    @staticmethod
    def params(p):
        return OrParams(*(int(p[f]) for f in ("n", "N", "k", "l", "Bgbit", "ks_t", "ks_basebit")))

    def external_product(self, p, bsk_row, acc, wide=False):
        P = self.params(p)
        acc = _i32(acc).copy()
        w = np.zeros(2 * acc.size, np.uint64) if wide else None
        self.L.or_external_product(ctypes.byref(P), _p(_i32(bsk_row)), _p(acc), _p(w))
        if wide:
            lo = w[0::2].astype(object)
            hi = w[1::2].astype(np.int64).astype(object)
            return acc, np.array([int(h) * (1 << 64) + int(l_) for l_, h in zip(lo, hi)], dtype=object)
        return acc

    def cmux_step(self, p, bsk_row, a, acc):
        P = self.params(p)
        acc = _i32(acc).copy()
        self.L.or_cmux_step(ctypes.byref(P), _p(_i32(bsk_row)), int(a), _p(acc))
        return acc

    def blind_rotate(self, p, bsk, bara, acc):
        P = self.params(p)
        acc = _i32(acc).copy()
        self.L.or_blind_rotate(ctypes.byref(P), _p(_i32(bsk)), _p(_i32(bara)), _p(acc))
        return acc

    def bootstrap_woks(self, p, bsk, mu, x):
        P = self.params(p)
        x = _i32(x)
        out = np.zeros((len(x), p["k"] * p["N"] + 1), np.int32)
        bsk = _i32(bsk)
        for g in range(len(x)):
            self.L.or_bootstrap_woks(ctypes.byref(P), _p(bsk), int(mu), _p(x[g]), _p(out[g]), None)
        return out

    def keyswitch(self, p, ksk, x):
        P = self.params(p)
        x = _i32(x)
        ksk = _i32(ksk)
        out = np.zeros((len(x), p["n"] + 1), np.int32)
        for g in range(len(x)):
            self.L.or_keyswitch(ctypes.byref(P), _p(ksk), _p(x[g]), _p(out[g]))
        return out

    def gate_prologue(self, n, code, ca, cb):
        ca, cb = _i32(ca), _i32(cb)
        out = np.zeros_like(ca)
        for g in range(len(ca)):
            self.L.or_gate_prologue(n, code, _p(ca[g]), _p(cb[g]), _p(out[g]))
        return out

    def gate(self, p, bsk, ksk, code, ca, cb=None, cc=None):
        P = self.params(p)
        ca = _i32(ca)
        cb = ca if cb is None else _i32(cb)
        cc = ca if cc is None else _i32(cc)
        bsk, ksk = _i32(bsk), _i32(ksk)
        out = np.zeros_like(ca)
        for g in range(len(ca)):
            self.L.or_gate(ctypes.byref(P), _p(bsk), _p(ksk), int(code), _p(ca[g]), _p(cb[g]), _p(cc[g]),
                           _p(out[g]))
        return out

    # ---- keys / encryption -----------------------------------------------------------------
    def keygen(self, p, ks_stdev=2**-15, bk_stdev=2**-25, seed=1):
        P = self.params(p)
        n, N, k, l = p["n"], p["N"], p["k"], p["l"]
        lk = np.zeros(n, np.int32)
        tk = np.zeros(k * N, np.int32)
        ksk = np.zeros((k * N, p["ks_t"], 1 << p["ks_basebit"], n + 1), np.int32)
        bsk = np.zeros((n, (k + 1) * l, k + 1, N), np.int32)
        self.L.or_keygen(ctypes.byref(P), ks_stdev, bk_stdev, seed, _p(lk), _p(tk), _p(ksk), _p(bsk))
        return lk, tk, ksk, bsk

    def encrypt_bits(self, key, bits, stdev=2**-15, seed=5):
        n = len(key)
        bits = np.asarray(bits)
        mus = np.where(bits != 0, 1 << 29, -(1 << 29)).astype(np.int32)
        out = np.zeros((len(bits), n + 1), np.int32)
        self.L.or_lwe_encrypt(n, _p(_i32(key)), _p(mus), stdev, seed, len(bits), _p(out))
        return out

    def phase(self, key, cts):
        cts = _i32(cts)
        key = _i32(key)
        return np.array([self.L.or_lwe_phase(len(key), _p(key), _p(c)) for c in cts], np.int32)

    def decrypt_bits(self, key, cts):
        return (self.phase(key, cts) > 0).astype(np.int32)


def torus_diff(a, b):
    """Signed difference a-b of Torus32 arrays, in Torus32 units (int64)."""
    d = np.asarray(a, np.int64) - np.asarray(b, np.int64)
    return ((d + 2**31) % 2**32) - 2**31
