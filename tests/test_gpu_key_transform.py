"""The FFT-domain bootstrapping key computed on the GPU (key_transform.cu) against numpy.

For sample key polynomials c: z_j = (c_j - i c_{j+M}) exp(-i pi j / N), Z = DFT_M(z), and slot
(r, t) must hold Z[slot_order[r, t]] / M.  FP64 keys within 1e-12 of the largest coefficient; the
split form checks both limbs c = hi * 2^S + lo within float rounding.
"""
import ctypes

import numpy as np
import pytest

import tfhe_b200 as tb

pytestmark = pytest.mark.gpu


def spectrum(poly, N):
    M = N // 2
    j = np.arange(M)
    z = (poly[:M].astype(np.float64) - 1j * poly[M:].astype(np.float64)) * np.exp(-1j * np.pi * j / N)
    return np.fft.fft(z) / M


@pytest.fixture(scope="module", params=["default", "large"])
def keys(request):
    p = tb.default_params() if request.param == "default" else tb.large_params()
    sk, ck = tb.keygen(p, seed=17)
    ck.to_device(0)
    bsk, _ = ck.export()
    return p, ck, bsk.reshape(-1, p.N)


def test_fp64_key_matches_numpy_fft(keys):
    p, ck, polys = keys
    got = ck.fft_key(tb.FP64)
    sf = tb.fft_slot_order(p.N)
    for idx in (0, 1, len(polys) // 2, len(polys) - 1):
        want = spectrum(polys[idx], p.N)[sf]                  # [8][N/16]
        g = got[idx][..., 0] + 1j * got[idx][..., 1]
        assert np.abs(g - want).max() <= 1e-12 * np.abs(want).max()


def test_split_key_limbs_match_numpy_fft(keys):
    p, ck, polys = keys
    S = int(tb.api.lib().tfheb_default_split_shift(ctypes.byref(p)))
    got = ck.fft_key(tb.SPLIT_FP32)                          # [poly][m][limb][t][4]
    sf = tb.fft_slot_order(p.N)
    for idx in (0, len(polys) - 1):
        c = polys[idx].astype(np.int64)
        lo = ((c + (1 << (S - 1))) & ((1 << S) - 1)) - (1 << (S - 1))
        hi = (c - lo) >> S
        for limb, part in ((0, hi), (1, lo)):
            want = spectrum(part, p.N)[sf]                   # [8][N/16]
            g = np.empty_like(want)
            for m in range(4):
                e = got[idx, m, limb]                        # [t][4] = re(2m), re(2m+1), im(2m), im(2m+1)
                g[2 * m] = e[:, 0] + 1j * e[:, 2]
                g[2 * m + 1] = e[:, 1] + 1j * e[:, 3]
            assert np.abs(g - want).max() <= 2e-7 * np.abs(want).max()
