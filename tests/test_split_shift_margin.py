"""The split form's high limb must round to the exact integer every time.  A numpy model of its FP32
arithmetic (complex64 folded negacyclic transforms of digit polynomials, multiply-accumulate against
FP32 spectra of high limbs over the (k+1)l rows, inverse transform) measures the error of the
high-limb sums against the exact integer products, at the shift S the library picks for each of the
reference's parameter sets; 1/2 must stay at least 12 sigma away (at 12 sigma a wrong rounding is
below 1e-30 per coefficient)."""
import ctypes

import numpy as np
import pytest

import tfhe_b200 as tb


def hi_limb_error(N, Bgbit, S, rows, trials, seed=1):
    rng = np.random.default_rng(seed)
    M = N // 2
    tw = np.exp(-1j * np.pi * np.arange(M) / N)

    def fwd(a, dt):  # z_j = (a_j - i a_{j+M}) exp(-i pi j / N), DFT of size M
        return np.fft.fft(((a[:M] - 1j * a[M:]) * tw).astype(dt)).astype(dt)

    errs = []
    for _ in range(trials):
        acc = np.zeros(M, np.complex64)
        exact = np.zeros(N, np.int64)
        for _ in range(rows):
            d = rng.integers(-(1 << (Bgbit - 1)), 1 << (Bgbit - 1), N)
            h = rng.integers(-(1 << (31 - S)), (1 << (31 - S)) + 1, N)
            acc = (acc + fwd(d.astype(np.float64), np.complex64)
                   * fwd(h.astype(np.float64), np.complex128).astype(np.complex64)).astype(np.complex64)
            full = np.convolve(d, h)
            prod = full[:N].copy()
            prod[:N - 1] -= full[N:]
            exact += prod
        z = np.fft.ifft(acc).astype(np.complex128) / tw
        errs.append(np.concatenate([z.real, -z.imag]) - exact)
    return float(np.sqrt(np.mean(np.concatenate(errs) ** 2)))


@pytest.mark.parametrize("which", ["default", "large", "lambda80"])
def test_high_limb_rounding_margin(which):
    p = {"default": tb.default_params, "large": tb.large_params, "lambda80": lambda: tb.default_params(80)}[which]()
    S = int(tb.api.lib().tfheb_default_split_shift(ctypes.byref(p)))
    sigma = hi_limb_error(p.N, p.Bgbit, S, (p.k + 1) * p.l, trials=2)
    assert 0.5 / sigma >= 12, f"S={S}: sigma {sigma:.4f}"
