"""Shared-memory bank model of the team FFT's exchanges (tfhe_b200/csrc/fft.cuh).

A thread of a team holds 8 points; between stages the team exchanges them through shared memory,
each exchange E (between stages E and E+1) under its own index map.  On B200 an 8-byte warp access
is served in two half-warp phases and a 16-byte one in four quarter-warp phases; a phase costs the
largest number of distinct words that fall on one bank (32 banks of 4 bytes), so the minimum is 2
wavefronts per 8-byte access and 4 per 16-byte access.  For 12 candidate FP32 maps of the 8*8*8 plan
this model reproduced the wavefronts ncu measured per instruction on B200.  The test mirrors the plans
and maps of fft.cuh and requires the minimum on every store and load of every exchange of the
8*8*4, 8*8*8 and 8*8*8*2 plans, for FP32 (float2) and FP64 (double2)."""
import pytest

PLANS = {256: [8, 8, 4], 512: [8, 8, 8], 1024: [8, 8, 8, 2]}


def positions(M, S):
    """Point index of register (c, n2) of each thread at stage S (TeamFft::pos)."""
    plan, NT = PLANS[M], M // 8
    L = M
    for s in range(S):
        L //= plan[s]
    r = plan[S]
    st = L // r
    out = []
    for c in range(8 // r):
        for n2 in range(r):
            row = []
            for t in range(NT):
                b = t + NT * c
                row.append((b // st) * L + b % st + st * n2)
            out.append(row)
    return out


def f32_index(M, E, p):  # exch_f32_map / exch_f32_index
    table = {256: [(5, 4, 6, 0, False), (2, 1, 6, 4, False)],
             512: [(5, 4, 6, 0, False), (3, 1, 4, 0, False)],
             1024: [(2, 0, 3, 0, False), (4, 2, 5, 0, False), (0, 0, 0, 0, True)]}
    s1, a, s2, b, swizzle = table[M][E]
    if swizzle:
        return p ^ ((p >> 2) & 7) ^ ((p >> 3) & 31)
    return p + a * (p >> s1) + b * (p >> s2)


def f64_index(M, E, p):  # Exch<double, M>::index
    return p + (p >> 3)


def wavefronts(elems, elem_words, phase_threads):
    total = 0
    for lo in range(0, len(elems), phase_threads):
        banks = {}
        for e in set(elems[lo:lo + phase_threads]):
            for w in range(elem_words):
                word = e * elem_words + w
                banks.setdefault(word % 32, set()).add(word)
        total += max(len(v) for v in banks.values())
    return total


@pytest.mark.parametrize("M", sorted(PLANS))
@pytest.mark.parametrize("form", ["f32", "f64"])
def test_every_exchange_access_takes_the_minimum_wavefronts(M, form):
    index, words, phase, minimum = ((f32_index, 2, 16, 2) if form == "f32" else (f64_index, 4, 8, 4))
    for E in range(len(PLANS[M]) - 1):
        idx = [index(M, E, p) for p in range(M)]
        assert len(set(idx)) == M  # one-to-one
        for S in (E, E + 1):  # the stores of stage E, the loads of stage E + 1
            for reg in positions(M, S):
                for w0 in range(0, len(reg), 32):
                    warp = [idx[p] for p in reg[w0:w0 + 32]]
                    assert wavefronts(warp, words, phase) == minimum, (M, E, S)


def test_the_model_penalises_the_bare_index():
    # the bare index p on stage 1 of the 8*8*8 plan: threads 8 apart sit 64 points apart, on the same
    # bank pair (ncu measured 6.5 wavefronts per access over all exchanges of this plan)
    reg = positions(512, 1)[0]
    assert wavefronts(reg[:32], 2, 16) > 2
