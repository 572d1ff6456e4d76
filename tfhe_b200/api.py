"""Python mirror of the engine's C ABI (include/tfhe_b200.h) over ctypes.

Mirrors the reference's gate-bootstrapping interface (tfhe_gate_bootstrapping_functions.h) on raw
int32 ciphertext arrays: keygen -> encrypt -> batched gates on the GPU -> decrypt.  Torch (or any
CUDA array with a data pointer) supplies device buffers for the *_device entry points.

The shared library is built in-tree (tfhe_b200/libtfhe_b200.so) by __graft_entry__.build();
importing this module never falls back to another implementation: if the library is missing,
loading fails loudly.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libtfhe_b200.so")

_V = ctypes.c_void_p
_I32 = ctypes.c_int32

NAND, OR, AND, XOR, XNOR, NOR, ANDNY, ANDYN, ORNY, ORYN, MUX, NOT, COPY = range(13)
GATE_NAMES = ["NAND", "OR", "AND", "XOR", "XNOR", "NOR", "ANDNY", "ANDYN", "ORNY", "ORYN", "MUX", "NOT", "COPY"]
FP64, SPLIT_FP32 = 0, 1


class TfhebError(RuntimeError):
    def __init__(self, msg, status=None):
        super().__init__(msg)
        self.status = status


TIMEOUT = 5


class Params(ctypes.Structure):
    _fields_ = [("n", _I32), ("N", _I32), ("k", _I32), ("l", _I32), ("Bgbit", _I32), ("ks_t", _I32),
                ("ks_basebit", _I32), ("ks_stdev", ctypes.c_double), ("bk_stdev", ctypes.c_double)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise TfhebError(f"{LIB_PATH} is missing: build it with __graft_entry__.build()")
        L = ctypes.CDLL(LIB_PATH)
        L.tfheb_last_error.restype = ctypes.c_char_p
        L.tfheb_kernel_launches.restype = ctypes.c_int64
        L.tfheb_keygen.argtypes = [ctypes.POINTER(Params), ctypes.c_uint64, ctypes.POINTER(_V), ctypes.POINTER(_V)]
        L.tfheb_encrypt.argtypes = [_V, _V, _I32, ctypes.c_uint64, _V]
        L.tfheb_decrypt.argtypes = [_V, _V, _I32, _V, _V]
        L.tfheb_cloud_key_to_device.argtypes = [_V, _I32, _I32, _I32]
        L.tfheb_cloud_key_import.argtypes = [ctypes.POINTER(Params), _V, _V, ctypes.POINTER(_V)]
        L.tfheb_secret_key_import.argtypes = [ctypes.POINTER(Params), _V, _V, ctypes.POINTER(_V)]
        L.tfheb_secret_key_export.argtypes = [_V, _V, _V]
        L.tfheb_cloud_key_export.argtypes = [_V, _V, _V]
        L.tfheb_secret_key_free.argtypes = [_V]
        L.tfheb_cloud_key_free.argtypes = [_V]
        L.tfheb_gate_batch.argtypes = [_V, _I32, _I32, _I32, _V, _V, _V, _V]
        L.tfheb_gate_batch_device.argtypes = [_V, _I32, _I32, _I32, _V, _V, _V, _V, _V]
        L.tfheb_bootstrap_woks_device.argtypes = [_V, _I32, _I32, _I32, _V, _V, _V]
        L.tfheb_bootstrap_device.argtypes = [_V, _I32, _I32, _I32, _V, _V, _V]
        L.tfheb_blind_rotate_device.argtypes = [_V, _I32, _I32, _I32, _V, _V, _V]
        L.tfheb_keyswitch_device.argtypes = [_V, _I32, _V, _V, _V]
        L.tfheb_synchronize.argtypes = [_V]
        L.tfheb_set_wait_timeout.argtypes = [_V, ctypes.c_uint64]
        L.tfheb_test_stall_key_stream.argtypes = [_V, _I32]
        L.tfheb_fft_slot_order.argtypes = [_I32, _V]
        L.tfheb_br_variants.argtypes = [_I32, _I32, _V, _V, _I32, _V]
        L.tfheb_cloud_key_br_variants.argtypes = [_V, _I32, _V, _V, _I32, _V]
        L.tfheb_cloud_key_br_plans.argtypes = [_V, _I32, _V, _I32, _V]
        L.tfheb_set_br_variant.argtypes = [_V, _I32, _I32]
        L.tfheb_autotune.argtypes = [_V, _I32, _I32, _V, _I32]
        L.tfheb_set_keyswitch_kernel.argtypes = [_V, _I32]
        L.tfheb_cloud_key_params.argtypes = [_V, ctypes.POINTER(Params)]
        L.tfheb_gate_batch_multi.argtypes = [_V, _I32, _I32, _I32, _I32, _V, _V, _V, _V]
        L.tfheb_cloud_key_fft_download.argtypes = [_V, _I32, _V, ctypes.c_size_t]
        _C = ctypes.c_char_p
        L.tfheb_params_save.argtypes = [_C, ctypes.POINTER(Params)]
        L.tfheb_params_load.argtypes = [_C, ctypes.POINTER(Params)]
        L.tfheb_cloud_key_save.argtypes = [_V, _C]
        L.tfheb_cloud_key_load.argtypes = [_C, ctypes.POINTER(_V)]
        L.tfheb_secret_keyset_save.argtypes = [_V, _V, _C]
        L.tfheb_secret_keyset_load.argtypes = [_C, ctypes.POINTER(_V), ctypes.POINTER(_V)]
        L.tfheb_ciphertexts_save.argtypes = [_C, ctypes.POINTER(Params), _I32, _V, _V]
        L.tfheb_ciphertexts_load.argtypes = [_C, ctypes.POINTER(Params), _I32, _V, _V]
        _lib = L
    return _lib


def _check(status, what):
    if status != 0:
        msg = lib().tfheb_last_error().decode(errors="replace")
        raise TfhebError(f"{what} failed with status {status}: {msg}", status)


def _p(a):
    if a is None:
        return None
    if isinstance(a, np.ndarray):
        return a.ctypes.data_as(_V)
    return _V(a.data_ptr())  # torch tensor


def _i32(a):
    return np.ascontiguousarray(a, dtype=np.int32)


def default_params(lam=128):
    p = Params()
    _check(lib().tfheb_default_params(lam, ctypes.byref(p)), "tfheb_default_params")
    return p


def large_params():
    p = Params()
    _check(lib().tfheb_large_params(ctypes.byref(p)), "tfheb_large_params")
    return p


def make_params(n, N, k, l, Bgbit, ks_t, ks_basebit, ks_stdev=2**-15, bk_stdev=2**-25):
    return Params(n, N, k, l, Bgbit, ks_t, ks_basebit, ks_stdev, bk_stdev)


def kernel_launches():
    return int(lib().tfheb_kernel_launches())


class SecretKey:
    def __init__(self, handle, params):
        self.h = _V(handle)
        self.params = params

    @classmethod
    def from_raw(cls, params, lwe_key, tlwe_key=None):
        h = _V()
        lk = _i32(lwe_key)
        tk = None if tlwe_key is None else _i32(tlwe_key)
        _check(lib().tfheb_secret_key_import(ctypes.byref(params), _p(lk), _p(tk), ctypes.byref(h)), "import")
        return cls(h.value, params)

    def export(self):
        p = self.params
        lk = np.zeros(p.n, np.int32)
        tk = np.zeros(p.k * p.N, np.int32)
        _check(lib().tfheb_secret_key_export(self.h, _p(lk), _p(tk)), "export")
        return lk, tk

    def encrypt(self, bits, seed=1):
        bits = _i32(bits)
        out = np.zeros((len(bits), self.params.n + 1), np.int32)
        _check(lib().tfheb_encrypt(self.h, _p(bits), len(bits), seed, _p(out)), "tfheb_encrypt")
        return out

    def decrypt(self, cts):
        cts = _i32(cts)
        bits = np.zeros(len(cts), np.int32)
        ph = np.zeros(len(cts), np.int32)
        _check(lib().tfheb_decrypt(self.h, _p(cts), len(cts), _p(bits), _p(ph)), "tfheb_decrypt")
        return bits, ph

    def free(self):
        if self.h:
            lib().tfheb_secret_key_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class CloudKey:
    """Cloud (evaluation) key: coefficient-domain keys on the host, FFT-domain keys on a GPU."""

    def __init__(self, handle, params):
        self.h = _V(handle)
        self.params = params

    @classmethod
    def from_raw(cls, params, bsk, ksk):
        h = _V()
        b, k = _i32(bsk), _i32(ksk)
        _check(lib().tfheb_cloud_key_import(ctypes.byref(params), _p(b), _p(k), ctypes.byref(h)), "import")
        return cls(h.value, params)

    def export(self):
        p = self.params
        bsk = np.zeros((p.n, (p.k + 1) * p.l, p.k + 1, p.N), np.int32)
        ksk = np.zeros((p.k * p.N, p.ks_t, 1 << p.ks_basebit, p.n + 1), np.int32)
        _check(lib().tfheb_cloud_key_export(self.h, _p(bsk), _p(ksk)), "export")
        return bsk, ksk

    def fft_key(self, precision):
        """The device FFT-domain bootstrapping key as stored (tfheb_cloud_key_fft_download)."""
        p = self.params
        polys = p.n * (p.k + 1) * p.l * (p.k + 1)
        nt = p.N // 16
        if precision == FP64:
            out = np.zeros((polys, 8, nt, 2), np.float64)
        else:
            out = np.zeros((polys, 4, 2, nt, 4), np.float32)
        _check(lib().tfheb_cloud_key_fft_download(self.h, precision, _p(out), out.nbytes),
               "tfheb_cloud_key_fft_download")
        return out

    def to_device(self, device=0, precisions=(FP64, SPLIT_FP32), split_shift=0):
        mask = 0
        for pr in precisions:
            mask |= 1 << pr
        _check(lib().tfheb_cloud_key_to_device(self.h, device, mask, split_shift), "tfheb_cloud_key_to_device")
        return self

    def gate(self, gate, a, b=None, c=None, precision=FP64):
        a = _i32(a)
        b = None if b is None else _i32(b)
        c = None if c is None else _i32(c)
        out = np.zeros_like(a)
        _check(lib().tfheb_gate_batch(self.h, gate, precision, len(a), _p(a), _p(b), _p(c), _p(out)),
               "tfheb_gate_batch")
        return out

    def gate_device(self, gate, d_a, d_b, d_c, d_out, count, precision=FP64, stream=None):
        _check(lib().tfheb_gate_batch_device(self.h, gate, precision, count, _p(d_a), _p(d_b), _p(d_c), _p(d_out),
                                             stream), "tfheb_gate_batch_device")

    def gate_mixed_device(self, gates, idx_a, idx_b, idx_c, out_idx, d_wires, num_wires, precision=FP64,
                          stream=None):
        """Mixed gate types over rows of a device wire array (tfheb_gate_batch_mixed_device); the index
        arrays are host arrays."""
        L = lib()
        L.tfheb_gate_batch_mixed_device.argtypes = [_V, _I32, _I32, _V, _V, _V, _V, _V, _V, _I32, _V]
        g = _i32(gates)
        ia, ib, ic, io = (_i32(x if x is not None else np.zeros(len(g))) for x in (idx_a, idx_b, idx_c, out_idx))
        _check(L.tfheb_gate_batch_mixed_device(self.h, precision, len(g), _p(g), _p(ia), _p(ib), _p(ic), _p(io),
                                               _p(d_wires), num_wires, stream), "tfheb_gate_batch_mixed_device")

    def bootstrap_woks_device(self, d_in, d_out, count, mu, precision=FP64, stream=None):
        _check(lib().tfheb_bootstrap_woks_device(self.h, precision, mu, count, _p(d_in), _p(d_out), stream),
               "tfheb_bootstrap_woks_device")

    def blind_rotate_device(self, d_bara, d_acc, count, nsteps, precision=FP64, stream=None):
        _check(lib().tfheb_blind_rotate_device(self.h, precision, count, nsteps, _p(d_bara), _p(d_acc), stream),
               "tfheb_blind_rotate_device")

    def keyswitch_device(self, d_in, d_out, count, stream=None):
        _check(lib().tfheb_keyswitch_device(self.h, count, _p(d_in), _p(d_out), stream), "tfheb_keyswitch_device")

    def br_variants(self, precision):
        """The autotuner's candidate variants for this key: (teams_per_cta, ring_depth) arrays."""
        cnt = ctypes.c_int32()
        G = np.zeros(16, np.int32)
        D = np.zeros(16, np.int32)
        _check(lib().tfheb_cloud_key_br_variants(self.h, precision, _p(G), _p(D), 16, ctypes.byref(cnt)),
               "tfheb_cloud_key_br_variants")
        return G[:cnt.value], D[:cnt.value]

    def br_plans(self, precision):
        """FFT plan of each candidate variant: 0 = one transform per thread, 1 = two transforms per
        thread on packed f32x2 with the digit spectra in tensor memory."""
        cnt = ctypes.c_int32()
        P = np.zeros(16, np.int32)
        _check(lib().tfheb_cloud_key_br_plans(self.h, precision, _p(P), 16, ctypes.byref(cnt)),
               "tfheb_cloud_key_br_plans")
        return P[:cnt.value]

    def autotune(self, precision, boots=4096):
        """Times every candidate blind-rotation variant (and the small-batch ones, for one-wave
        batches); returns [{teams_per_cta, ring_depth, plan, ms}] of the candidates."""
        G, D = self.br_variants(precision)
        P = self.br_plans(precision)
        ms = np.zeros(len(G), np.float64)
        _check(lib().tfheb_autotune(self.h, precision, boots, _p(ms), len(G)), "tfheb_autotune")
        return [{"teams_per_cta": int(g), "ring_depth": int(d), "plan": int(pl), "ms": float(m)}
                for g, d, pl, m in zip(G, D, P, ms)]

    def set_br_variant(self, precision, variant):
        _check(lib().tfheb_set_br_variant(self.h, precision, variant), "tfheb_set_br_variant")

    def set_keyswitch_kernel(self, which):
        """0 = default, 1 = one CTA per sample, 2 = tiled, 3 = register-key, 4 = tensor-core
        (bit-identical results)."""
        _check(lib().tfheb_set_keyswitch_kernel(self.h, which), "tfheb_set_keyswitch_kernel")

    def set_wait_timeout(self, seconds):
        _check(lib().tfheb_set_wait_timeout(self.h, ctypes.c_uint64(int(seconds * 1e9))), "tfheb_set_wait_timeout")

    def test_stall_key_stream(self, stall=True):
        _check(lib().tfheb_test_stall_key_stream(self.h, 1 if stall else 0), "tfheb_test_stall_key_stream")

    def synchronize(self):
        _check(lib().tfheb_synchronize(self.h), "tfheb_synchronize")

    def free(self):
        if self.h:
            lib().tfheb_cloud_key_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def keygen(params, seed=1):
    sk, ck = _V(), _V()
    _check(lib().tfheb_keygen(ctypes.byref(params), seed, ctypes.byref(sk), ctypes.byref(ck)), "tfheb_keygen")
    return SecretKey(sk.value, params), CloudKey(ck.value, params)


def gate_batch_multi(cks, gate, a, b=None, c=None, precision=FP64):
    """One batch of gates sharded across cloud keys on several GPUs (tfheb_gate_batch_multi)."""
    a = _i32(a)
    b = None if b is None else _i32(b)
    c = None if c is None else _i32(c)
    out = np.zeros_like(a)
    arr = (_V * len(cks))(*[k.h for k in cks])
    _check(lib().tfheb_gate_batch_multi(ctypes.cast(arr, _V), len(cks), gate, precision, len(a), _p(a), _p(b),
                                        _p(c), _p(out)), "tfheb_gate_batch_multi")
    return out


# ---- files in the reference's format (tfhe_io.cpp) -------------------------------------------

def _path(path):
    return os.fsencode(path)


def save_params(path, params):
    _check(lib().tfheb_params_save(_path(path), ctypes.byref(params)), "tfheb_params_save")


def load_params(path):
    p = Params()
    _check(lib().tfheb_params_load(_path(path), ctypes.byref(p)), "tfheb_params_load")
    return p


def _cloud_params(h):
    p = Params()
    _check(lib().tfheb_cloud_key_params(h, ctypes.byref(p)), "tfheb_cloud_key_params")
    return p


def save_cloud_keyset(path, ck):
    _check(lib().tfheb_cloud_key_save(ck.h, _path(path)), "tfheb_cloud_key_save")


def load_cloud_keyset(path):
    h = _V()
    _check(lib().tfheb_cloud_key_load(_path(path), ctypes.byref(h)), "tfheb_cloud_key_load")
    return CloudKey(h.value, _cloud_params(h))


def save_secret_keyset(path, sk, ck):
    _check(lib().tfheb_secret_keyset_save(sk.h, ck.h, _path(path)), "tfheb_secret_keyset_save")


def load_secret_keyset(path):
    s, c = _V(), _V()
    _check(lib().tfheb_secret_keyset_load(_path(path), ctypes.byref(s), ctypes.byref(c)), "tfheb_secret_keyset_load")
    p = _cloud_params(c)
    return SecretKey(s.value, p), CloudKey(c.value, p)


def save_ciphertexts(path, params, cts, variances=None):
    cts = _i32(cts).reshape(-1, params.n + 1)
    v = None if variances is None else np.ascontiguousarray(variances, dtype=np.float64)
    _check(lib().tfheb_ciphertexts_save(_path(path), ctypes.byref(params), len(cts), _p(cts), _p(v)),
           "tfheb_ciphertexts_save")


def load_ciphertexts(path, params, count):
    out = np.zeros((count, params.n + 1), np.int32)
    v = np.zeros(count, np.float64)
    _check(lib().tfheb_ciphertexts_load(_path(path), ctypes.byref(params), count, _p(out), _p(v)),
           "tfheb_ciphertexts_load")
    return out, v


class Netlist:
    """Levelled gate netlist on the GPU (tfheb_netlist_*): wires 0..num_inputs-1 are inputs, gate g
    writes wire num_inputs+g."""

    def __init__(self, ck, num_inputs, gates, in_a, in_b=None, in_c=None):
        L = lib()
        L.tfheb_netlist_create.argtypes = [_V, _I32, _I32, _V, _V, _V, _V, ctypes.POINTER(_V)]
        L.tfheb_netlist_info.argtypes = [_V, _V, _V]
        L.tfheb_netlist_run.argtypes = [_V, _I32, _V, _I32, _V]
        L.tfheb_netlist_free.argtypes = [_V]
        self.ck = ck
        self.num_inputs = int(num_inputs)
        self.gates = _i32(gates)
        g = len(self.gates)
        self._a = _i32(in_a)
        self._b = _i32(in_b if in_b is not None else np.zeros(g))
        self._c = _i32(in_c if in_c is not None else np.zeros(g))
        h = _V()
        _check(L.tfheb_netlist_create(ck.h, self.num_inputs, g, _p(self.gates), _p(self._a), _p(self._b),
                                      _p(self._c), ctypes.byref(h)), "tfheb_netlist_create")
        self.h = h

    def info(self):
        lv, w = ctypes.c_int32(), ctypes.c_int32()
        _check(lib().tfheb_netlist_info(self.h, ctypes.byref(lv), ctypes.byref(w)), "tfheb_netlist_info")
        return lv.value, w.value

    def run(self, d_wires, precision=FP64, use_graph=True, stream=None):
        _check(lib().tfheb_netlist_run(self.h, precision, _p(d_wires), 1 if use_graph else 0, stream),
               "tfheb_netlist_run")

    def free(self):
        if self.h:
            lib().tfheb_netlist_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class NetlistMulti:
    """A netlist sharded across several cloud keys / GPUs (tfheb_netlist_multi_*), evaluated from and
    to a host wire array."""

    def __init__(self, cks, num_inputs, gates, in_a, in_b=None, in_c=None):
        L = lib()
        L.tfheb_netlist_multi_create.argtypes = [_V, _I32, _I32, _I32, _V, _V, _V, _V, ctypes.POINTER(_V)]
        L.tfheb_netlist_multi_run.argtypes = [_V, _I32, _V]
        L.tfheb_netlist_multi_free.argtypes = [_V]
        self.cks = list(cks)
        self.num_inputs = int(num_inputs)
        self.gates = _i32(gates)
        g = len(self.gates)
        self._a = _i32(in_a)
        self._b = _i32(in_b if in_b is not None else np.zeros(g))
        self._c = _i32(in_c if in_c is not None else np.zeros(g))
        arr = (_V * len(self.cks))(*[k.h for k in self.cks])
        h = _V()
        self.h = None
        _check(L.tfheb_netlist_multi_create(ctypes.cast(arr, _V), len(self.cks), self.num_inputs, g, _p(self.gates),
                                            _p(self._a), _p(self._b), _p(self._c), ctypes.byref(h)),
               "tfheb_netlist_multi_create")
        self.h = h

    def run(self, inputs, precision=FP64):
        """inputs: [num_inputs][n+1] ciphertexts; returns the wire array [num_inputs+num_gates][n+1]."""
        inputs = _i32(inputs)
        wires = np.zeros((self.num_inputs + len(self.gates), inputs.shape[1]), np.int32)
        wires[:self.num_inputs] = inputs
        _check(lib().tfheb_netlist_multi_run(self.h, precision, _p(wires)), "tfheb_netlist_multi_run")
        return wires

    def free(self):
        if self.h:
            lib().tfheb_netlist_multi_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def random_netlist(rng, levels, width_lo, width_hi, mix=None, first_width=None):
    """Seeded layered netlist: level widths uniform in [width_lo, width_hi]; gate types drawn with
    the probabilities `mix` ({code: p}); every operand uniform over the previous two levels.
    Returns (num_inputs, gates, in_a, in_b, in_c)."""
    mix = mix or {NAND: 0.40, XOR: 0.20, AND: 0.15, OR: 0.15, MUX: 0.10}
    codes = np.array(list(mix.keys()))
    probs = np.array(list(mix.values()), dtype=np.float64)
    probs /= probs.sum()
    w0 = first_width or int(rng.integers(width_lo, width_hi + 1))
    spans = [(0, w0)]  # wire ranges of each level
    gates, ia, ib, ic = [], [], [], []
    nxt = w0
    for _ in range(levels):
        w = int(rng.integers(width_lo, width_hi + 1))
        lo = spans[-2][0] if len(spans) >= 2 else spans[-1][0]
        hi = spans[-1][1]
        gates.append(rng.choice(codes, size=w, p=probs))
        ia.append(rng.integers(lo, hi, size=w))
        ib.append(rng.integers(lo, hi, size=w))
        ic.append(rng.integers(lo, hi, size=w))
        spans.append((nxt, nxt + w))
        nxt += w
    return (w0, np.concatenate(gates).astype(np.int32), np.concatenate(ia).astype(np.int32),
            np.concatenate(ib).astype(np.int32), np.concatenate(ic).astype(np.int32))


def eval_plain(num_inputs, gates, in_a, in_b, in_c, input_bits):
    """Plaintext evaluation of a netlist (the truth the decrypted wires must equal)."""
    wires = np.zeros(num_inputs + len(gates), np.int32)
    wires[:num_inputs] = input_bits
    for g, code in enumerate(gates):
        a, b, c = wires[in_a[g]], wires[in_b[g]], wires[in_c[g]]
        wires[num_inputs + g] = [1 - (a & b), a | b, a & b, a ^ b, 1 - (a ^ b), 1 - (a | b), (1 - a) & b,
                                 a & (1 - b), (1 - a) | b, a | (1 - b), b if a else c, 1 - a, a][code]
    return wires


def br_variants(N, precision):
    cnt = ctypes.c_int32()
    G = np.zeros(16, np.int32)
    D = np.zeros(16, np.int32)
    _check(lib().tfheb_br_variants(N, precision, _p(G), _p(D), 16, ctypes.byref(cnt)), "tfheb_br_variants")
    return G[:cnt.value], D[:cnt.value]


def fft_slot_order(N):
    out = np.zeros(N // 2, np.int32)
    _check(lib().tfheb_fft_slot_order(N, _p(out)), "tfheb_fft_slot_order")
    return out.reshape(8, N // 16)
