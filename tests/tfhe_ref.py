"""ctypes bindings for the reference library shim (oracle/_ref/libtfhe_ref_shim.so).

Test infrastructure: drives the unmodified reference (tfhe v1.1, spqlios-fma) built from its own
sources by oracle/ref.mk.  Used to generate golden vectors, to run the reference live on identical
inputs when its build is present, and as the timed CPU baseline.
"""
import ctypes
import os

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_DIR = os.path.join(ROOT, "oracle", "_ref")
SHIM = os.path.join(REF_DIR, "libtfhe_ref_shim.so")

_V = ctypes.c_void_p
_I = ctypes.c_int32


def _p(a):
    return None if a is None else a.ctypes.data_as(_V)


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


class RefKeys:
    """A reference TFheGateBootstrappingSecretKeySet plus raw accessors."""

    def __init__(self, lib, handle):
        self.lib = lib
        self.h = _V(handle)
        d = np.zeros(8, np.int32)
        lib.rs_dims(self.h, _p(d))
        self.n, self.N, self.k, self.l, self.Bgbit, self.ks_t, self.ks_basebit, self.kpl = map(int, d)

    def params(self):
        return dict(n=self.n, N=self.N, k=self.k, l=self.l, Bgbit=self.Bgbit,
                    ks_t=self.ks_t, ks_basebit=self.ks_basebit)

    def export(self, bsk=True, ksk=True):
        n, N, k = self.n, self.N, self.k
        lk = np.zeros(n, np.int32)
        tk = np.zeros(k * N, np.int32)
        kk = np.zeros((k * N, self.ks_t, 1 << self.ks_basebit, n + 1), np.int32) if ksk else None
        bk = np.zeros((n, self.kpl, k + 1, N), np.int32) if bsk else None
        self.lib.rs_export(self.h, _p(lk), _p(tk), _p(kk), _p(bk))
        return lk, tk, kk, bk

    def encrypt(self, bits):
        bits = _i32(bits)
        out = np.zeros((len(bits), self.n + 1), np.int32)
        self.lib.rs_encrypt(self.h, len(bits), _p(bits), _p(out))
        return out

    def decrypt(self, cts):
        cts = _i32(cts)
        bits = np.zeros(len(cts), np.int32)
        ph = np.zeros(len(cts), np.int32)
        self.lib.rs_decrypt(self.h, len(cts), _p(cts), _p(bits), _p(ph))
        return bits, ph

    def gate(self, code, a, b=None, c=None):
        a = _i32(a)
        b = None if b is None else _i32(b)
        c = None if c is None else _i32(c)
        out = np.zeros_like(a)
        self.lib.rs_gate(self.h, code, len(a), _p(a), _p(b), _p(c), _p(out))
        return out

    def bootstrap_woks(self, mu, x):
        x = _i32(x)
        out = np.zeros((len(x), self.k * self.N + 1), np.int32)
        self.lib.rs_bootstrap_woks(self.h, mu, len(x), _p(x), _p(out))
        return out

    def keyswitch(self, x, with_variance=False):
        x = _i32(x)
        out = np.zeros((len(x), self.n + 1), np.int32)
        var = np.zeros(len(x), np.float64) if with_variance else None
        self.lib.rs_keyswitch(self.h, len(x), _p(x), _p(out), _p(var))
        return (out, var) if with_variance else out

    def extern_product(self, i, b, b_var):
        """tGswExternProduct with the coefficient-domain key sample i: (result, its variance)."""
        b = _i32(b)
        out = np.zeros_like(b)
        var = ctypes.c_double()
        self.lib.rs_extern_product(self.h, i, _p(b), ctypes.c_double(b_var), _p(out), ctypes.byref(var))
        return out, var.value

    def extern_mul(self, i, acc):
        acc = _i32(acc).copy()
        self.lib.rs_extern_mul(self.h, i, _p(acc))
        return acc

    def bench_gates(self, code, threads, per_thread, a, b, c, out):
        return self.lib.rs_bench_gates(self.h, code, threads, per_thread, _p(a), _p(b), _p(c), _p(out))

    # the reference's own file format (tfhe_io.cpp FILE* functions)
    def save_params(self, path):
        assert self.lib.rs_save_params(self.h, path.encode()) == 0

    def save_secret_keyset(self, path):
        assert self.lib.rs_save_secret_keyset(self.h, path.encode()) == 0

    def save_cloud_keyset(self, path):
        assert self.lib.rs_save_cloud_keyset(self.h, path.encode()) == 0

    def save_ciphertexts(self, path, cts, variances):
        cts = _i32(cts)
        v = np.ascontiguousarray(variances, dtype=np.float64)
        assert self.lib.rs_save_ciphertexts(self.h, path.encode(), len(cts), _p(cts), _p(v)) == 0

    def load_ciphertexts(self, path, count):
        out = np.zeros((count, self.n + 1), np.int32)
        v = np.zeros(count, np.float64)
        assert self.lib.rs_load_ciphertexts(self.h, path.encode(), count, _p(out), _p(v)) == 0
        return out, v

    def free(self):
        if self.h is not None:
            self.lib.rs_free(self.h)
            self.h = None


class RefLib:
    _inst = None

    def __init__(self, path):
        L = ctypes.CDLL(path)
        L.rs_keygen.restype = _V
        L.rs_keygen.argtypes = [ctypes.c_int] * 8 + [ctypes.c_double] * 2 + [ctypes.c_uint32]
        L.rs_bench_gates.restype = ctypes.c_double
        L.rs_bench_gates.argtypes = [_V, ctypes.c_int, _I, _I, _V, _V, _V, _V]
        L.rs_dtot32.argtypes = [ctypes.c_double]
        L.rs_load_secret_keyset.restype = _V
        L.rs_load_secret_keyset.argtypes = [ctypes.c_char_p]
        for f in ("rs_save_params", "rs_save_secret_keyset", "rs_save_cloud_keyset"):
            getattr(L, f).argtypes = [_V, ctypes.c_char_p]
        L.rs_save_ciphertexts.argtypes = [_V, ctypes.c_char_p, _I, _V, _V]
        L.rs_load_ciphertexts.argtypes = [_V, ctypes.c_char_p, _I, _V, _V]
        self.L = L

    @classmethod
    def available(cls):
        return os.path.exists(SHIM)

    @classmethod
    def load(cls, required=False):
        if cls._inst is None:
            if not os.path.exists(SHIM):
                if required:
                    raise RuntimeError(f"reference build missing: {SHIM} (run make -f oracle/ref.mk)")
                return None
            cls._inst = RefLib(SHIM)
        return cls._inst

    def keygen(self, custom=None, ks_stdev=2**-15, bk_stdev=2**-25, seed=1):
        if custom is None:
            h = self.L.rs_keygen(0, 0, 0, 0, 0, 0, 0, 0, 0.0, 0.0, seed)
        else:
            p = custom
            h = self.L.rs_keygen(1, p["n"], p["N"], p["k"], p["l"], p["Bgbit"], p["ks_t"], p["ks_basebit"],
                                 ks_stdev, bk_stdev, seed)
        return RefKeys(self.L, h)

    def load_secret_keyset(self, path):
        """new_tfheGateBootstrappingSecretKeySet_fromFile on a file (parameters from the file)."""
        h = self.L.rs_load_secret_keyset(os.fsencode(path))
        assert h, f"reference could not open {path}"
        return RefKeys(self.L, h)

    def modswitch_from(self, phase, msize):
        return self.L.rs_modswitch_from(phase, msize)

    def modswitch_to(self, mu, msize):
        return self.L.rs_modswitch_to(mu, msize)

    def decompose(self, N, l, bgbit, poly):
        out = np.zeros((l, N), np.int32)
        self.L.rs_decompose(N, l, bgbit, _p(_i32(poly)), _p(out))
        return out

    def rotate(self, N, a, minus_one, poly):
        out = np.zeros(N, np.int32)
        self.L.rs_rotate(N, a, 1 if minus_one else 0, _p(_i32(poly)), _p(out))
        return out

    def extract(self, N, k, tlwe):
        out = np.zeros(k * N + 1, np.int32)
        self.L.rs_extract(N, k, _p(_i32(tlwe)), _p(out))
        return out

    def poly_mult(self, kind, N, ipoly, tpoly):
        out = np.zeros(N, np.int32)
        self.L.rs_poly_mult(kind, N, _p(_i32(ipoly)), _p(_i32(tpoly)), _p(out))
        return out
