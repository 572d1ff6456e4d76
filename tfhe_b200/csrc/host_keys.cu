// host_keys.cu -- host-side key material: generation, encryption, the FFT twiddle tables and the
// slot order of the kernels' spectra (the FFT-domain key itself is computed on the GPU,
// key_transform.cu).
//
// Key generation follows the reference's distributions and structure
//   lweKeyGen / tLweKeyGen            lwe-functions.cpp:20-26, tlwe-functions.cpp:15-23
//   lweCreateKeySwitchKey             lwe-keyswitch-functions.cpp:163-215 (centred noise, h=0 rows zero)
//   tfhe_createLweBootstrappingKey    lwe-bootstrapping-functions.cpp:185-217 (tGswSymEncryptInt per s_i)
// with exact products (the TLWE key is binary, so b += s*a is a sum of signed rotations of a) and a
// self-contained seeded generator, so keys are reproducible at every ring degree.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <functional>
#include <cstring>
#include <thread>
#include <vector>

#include "fft.cuh"
#include "internal.h"

namespace tfheb {

// ---- numerics (numeric-functions.cpp:33-76) --------------------------------------------------

int32_t modswitch_to_torus32(int32_t mu, int32_t msize) {
    const uint64_t interv = ((UINT64_C(1) << 63) / (uint64_t)msize) * 2;
    return (int32_t)(uint32_t)(((uint64_t)(int64_t)mu * interv) >> 32);
}

int32_t modswitch_from_torus32(int32_t phase, int32_t msize) {
    const uint64_t interv = ((UINT64_C(1) << 63) / (uint64_t)msize) * 2;
    const uint64_t phase64 = ((uint64_t)(uint32_t)phase << 32) + interv / 2;
    return (int32_t)(phase64 / interv);
}

int32_t double_to_torus32(double d) {
    const double frac = d - (double)(int64_t)d;
    return (int32_t)(uint32_t)(uint64_t)(int64_t)(frac * 4294967296.0);
}

// the nearest multiple of 1/msize (approxPhase, numeric-functions.cpp:45-53)
int32_t approx_phase(int32_t phase, int32_t msize) {
    const uint64_t interv = ((UINT64_C(1) << 63) / (uint64_t)msize) * 2;
    uint64_t p64 = ((uint64_t)(uint32_t)phase << 32) + interv / 2;
    p64 -= p64 % interv;
    return (int32_t)(uint32_t)(p64 >> 32);
}

// ---- generator -------------------------------------------------------------------------------

namespace {
struct Rng {
    uint64_t s[4];
    bool spare_ok = false;
    double spare = 0;
    explicit Rng(uint64_t seed) {
        for (auto &w : s) {  // splitmix64 expansion
            uint64_t z = (seed += UINT64_C(0x9E3779B97F4A7C15));
            z = (z ^ (z >> 30)) * UINT64_C(0xBF58476D1CE4E5B9);
            z = (z ^ (z >> 27)) * UINT64_C(0x94D049BB133111EB);
            w = z ^ (z >> 31);
        }
    }
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {  // xoshiro256**
        const uint64_t r = rotl(s[1] * 5, 7) * 9, t = s[1] << 17;
        s[2] ^= s[0];
        s[3] ^= s[1];
        s[1] ^= s[2];
        s[0] ^= s[3];
        s[2] ^= t;
        s[3] = rotl(s[3], 45);
        return r;
    }
    int32_t torus() { return (int32_t)(uint32_t)(next() >> 32); }
    int32_t bit() { return (int32_t)(next() >> 63); }
    double normal() {  // Marsaglia polar
        if (spare_ok) {
            spare_ok = false;
            return spare;
        }
        double u, v, q;
        do {
            u = (double)(next() >> 11) * 0x1.0p-53 * 2.0 - 1.0;
            v = (double)(next() >> 11) * 0x1.0p-53 * 2.0 - 1.0;
            q = u * u + v * v;
        } while (q >= 1.0 || q == 0.0);
        const double m = std::sqrt(-2.0 * std::log(q) / q);
        spare = v * m;
        spare_ok = true;
        return u * m;
    }
};

// b += s * a in Z_{2^32}[X]/(X^N+1) for a binary polynomial s
void add_binary_product(int N, const int32_t *s, const int32_t *a, uint32_t *b) {
    for (int j = 0; j < N; j++) {
        if (!s[j]) continue;
        const uint32_t *ua = reinterpret_cast<const uint32_t *>(a);
        for (int i = 0; i < N - j; i++) b[i + j] += ua[i];
        for (int i = N - j; i < N; i++) b[i + j - N] -= ua[i];
    }
}

void parallel_for(int count, const std::function<void(int)> &fn) {
    unsigned hw = std::thread::hardware_concurrency();
    const int nt = (int)std::max(1u, std::min(hw ? hw : 1u, 32u));
    std::vector<std::thread> pool;
    std::atomic<int> next{0};
    for (int w = 0; w < nt; w++)
        pool.emplace_back([&]() {
            for (int i; (i = next.fetch_add(1)) < count;) fn(i);
        });
    for (auto &th : pool) th.join();
}
}  // namespace

void keygen(const tfheb_params &p, uint64_t seed, SecretKey &sk, CloudKey &ck) {
    const int n = p.n, N = p.N, k = p.k, l = p.l, kN = p.k * p.N, t = p.ks_t;
    const int base = 1 << p.ks_basebit, kpl = (k + 1) * l;
    sk.p = p;
    ck.p = p;
    Rng rng(seed);
    sk.lwe_key.resize(n);
    sk.tlwe_key.resize(kN);
    for (auto &v : sk.lwe_key) v = rng.bit();
    for (auto &v : sk.tlwe_key) v = rng.bit();

    // keyswitching key: extracted key (= TLWE key coefficients) -> LWE key
    const int64_t sizeks = (int64_t)kN * t * (base - 1);
    std::vector<double> noise(sizeks);
    double mean = 0;
    for (auto &e : noise) {
        e = rng.normal() * p.ks_stdev;
        mean += e;
    }
    mean /= (double)sizeks;
    ck.ksk.assign((size_t)kN * t * base * (n + 1), 0);
    int64_t idx = 0;
    for (int i = 0; i < kN; i++)
        for (int j = 0; j < t; j++)
            for (int h = 1; h < base; h++) {
                int32_t *row = ck.ksk.data() + (((size_t)i * t + j) * base + h) * (n + 1);
                const uint32_t mess = (uint32_t)(sk.tlwe_key[i] * h) << (32 - (j + 1) * p.ks_basebit);
                uint32_t b = mess + (uint32_t)double_to_torus32(noise[idx++] - mean);
                for (int c = 0; c < n; c++) {
                    row[c] = rng.torus();
                    b += (uint32_t)row[c] * (uint32_t)sk.lwe_key[c];
                }
                row[n] = (int32_t)b;
            }

    // bootstrapping key: TGSW(s_i) rows, independent generator per i (parallel)
    ck.bsk_coef.assign((size_t)n * kpl * (k + 1) * N, 0);
    const uint64_t bsk_seed = rng.next();
    parallel_for(n, [&](int i) {
        Rng r(bsk_seed ^ (UINT64_C(0xD1B54A32D192ED03) * (uint64_t)(i + 1)));
        for (int pr = 0; pr < kpl; pr++) {
            int32_t *row = ck.bsk_coef.data() + ((size_t)i * kpl + pr) * (k + 1) * N;
            uint32_t *b = reinterpret_cast<uint32_t *>(row + (size_t)k * N);
            for (int j = 0; j < N; j++) b[j] = (uint32_t)double_to_torus32(r.normal() * p.bk_stdev);
            for (int u = 0; u < k; u++) {
                int32_t *a = row + (size_t)u * N;
                for (int j = 0; j < N; j++) a[j] = r.torus();
                add_binary_product(N, sk.tlwe_key.data() + (size_t)u * N, a, b);
            }
            // + s_i * h_q on component (pr / l), coefficient 0 (tgsw-functions.cpp:111-122)
            const int bloc = pr / l, q = pr % l;
            const uint32_t hq = 1u << (32 - (q + 1) * p.Bgbit);
            row[(size_t)bloc * N] = (int32_t)((uint32_t)row[(size_t)bloc * N] + (uint32_t)sk.lwe_key[i] * hq);
        }
    });
}

void encrypt(const SecretKey &sk, const int32_t *bits, int32_t count, uint64_t seed, int32_t *out) {
    const int n = sk.p.n;
    const uint32_t mu = (uint32_t)modswitch_to_torus32(1, 8);
    Rng rng(seed);
    for (int g = 0; g < count; g++) {
        int32_t *ct = out + (size_t)g * (n + 1);
        uint32_t b = (bits[g] ? mu : 0u - mu) + (uint32_t)double_to_torus32(rng.normal() * sk.p.ks_stdev);
        for (int i = 0; i < n; i++) {
            ct[i] = rng.torus();
            b += (uint32_t)ct[i] * (uint32_t)sk.lwe_key[i];
        }
        ct[n] = (int32_t)b;
    }
}

// LWE encryptions of torus messages under key[n] with noise stdev (lweSymEncrypt, lwe-functions.cpp:33-44)
void encrypt_torus(int n, const int32_t *key, const int32_t *mu, int32_t count, double stdev, uint64_t seed,
                   int32_t *out) {
    Rng rng(seed);
    for (int g = 0; g < count; g++) {
        int32_t *ct = out + (size_t)g * (n + 1);
        uint32_t b = (uint32_t)mu[g] + (uint32_t)double_to_torus32(rng.normal() * stdev);
        for (int i = 0; i < n; i++) {
            ct[i] = rng.torus();
            b += (uint32_t)ct[i] * (uint32_t)key[i];
        }
        ct[n] = (int32_t)b;
    }
}

int32_t phase(const SecretKey &sk, const int32_t *ct) {
    uint32_t axs = 0;
    for (int i = 0; i < sk.p.n; i++) axs += (uint32_t)ct[i] * (uint32_t)sk.lwe_key[i];
    return (int32_t)((uint32_t)ct[sk.p.n] - axs);
}

// ---- FFT layout ------------------------------------------------------------------------------

namespace {
template <int M>
void slot_freq_m(std::vector<int32_t> &out) {
    constexpr int NT = M / kR, NS = FftPlan<M>::NS;
    constexpr int rl = FftPlan<M>::radix(NS - 1);
    out.assign(kR * NT, 0);
    for (int t = 0; t < NT; t++)
        for (int reg = 0; reg < kR; reg++) {
            const int c = reg / rl, n2 = reg % rl;
            const int L = stage_len<M>(NS - 1), st = L / rl;
            const int b = t + NT * c, q = b / st, n1 = b - q * st;
            const int p = q * L + n1 + st * n2;  // last-stage position
            int kf = 0, mul = 1;
            for (int s = 0; s < NS; s++) {  // mixed-radix digit reversal
                const int r = FftPlan<M>::radix(s);
                const int d = (p / stage_len<M>(s + 1)) % r;
                kf += d * mul;
                mul *= r;
            }
            out[reg * NT + t] = kf;
        }
}

template <int M>
void tables_m(std::vector<double> &tab) {
    constexpr int NT = M / kR, NS = FftPlan<M>::NS, N = 2 * M;
    const int tw = tw_offset<M>(NS);
    tab.assign(2 * (size_t)tw, 0.0);
    auto put = [&](int idx, long double ang_over_pi) {
        tab[2 * idx] = (double)std::cos((long double)M_PI * ang_over_pi);
        tab[2 * idx + 1] = (double)std::sin((long double)M_PI * ang_over_pi);
    };
    // stage 0: exp(-i pi t / N) * W_M^{t k2} = exp(-i pi t (1 + 4 k2) / N), k2 in [0, 8)
    for (int k2 = 0; k2 < kR; k2++)
        for (int t = 0; t < NT; t++) {
            const long e = ((long)t * (1 + 4 * k2)) % (2 * N);
            put(k2 * NT + t, -(long double)e / (long double)N);
        }
    for (int s = 1; s < NS; s++) {
        const int L = stage_len<M>(s), r = FftPlan<M>::radix(s), st = L / r;
        const int off = tw_offset<M>(s);
        for (int k2 = 1; k2 < r; k2++)
            for (int n1 = 0; n1 < st; n1++) {
                const long e = ((long)n1 * k2) % L;  // W_L^e = exp(-2 pi i e / L)
                put(off + (k2 - 1) * st + n1, -2.0L * (long double)e / (long double)L);
            }
    }
}

// The FP32 table in float4 pairs (tw4_offset): the FP64 factors rounded to float.
template <int M>
void tables_f32_m(std::vector<float> &tf) {
    std::vector<double> tab;
    tables_m<M>(tab);
    constexpr int NT = M / kR, NS = FftPlan<M>::NS;
    tf.assign(4 * (size_t)tw4_offset<M>(NS), 0.f);
    auto pair = [&](int at4, int i0, int i1) {  // complex entries i0, i1 of the FP64 table (-1: zero pad)
        float *o = &tf[4 * (size_t)at4];
        if (i0 >= 0) o[0] = (float)tab[2 * i0], o[1] = (float)tab[2 * i0 + 1];
        if (i1 >= 0) o[2] = (float)tab[2 * i1], o[3] = (float)tab[2 * i1 + 1];
    };
    for (int q = 0; q < kR / 2; q++)
        for (int t = 0; t < NT; t++) pair(q * NT + t, (2 * q) * NT + t, (2 * q + 1) * NT + t);
    for (int s = 1; s < NS; s++) {
        const int L = stage_len<M>(s), r = FftPlan<M>::radix(s), st = L / r;
        const int off = tw_offset<M>(s), off4 = tw4_offset<M>(s);
        for (int q = 0; q < r / 2; q++)
            for (int n1 = 0; n1 < st; n1++) {
                const int k0 = 2 * q + 1, k1 = 2 * q + 2;
                pair(off4 + q * st + n1, off + (k0 - 1) * st + n1, k1 < r ? off + (k1 - 1) * st + n1 : -1);
            }
    }
}

template <int M>
void tables_f32_paired_m(std::vector<float> &tf) {
    std::vector<double> tab;
    tables_m<M>(tab);
    const size_t n = tab.size() / 2;
    tf.assign(4 * n, 0.f);
    for (size_t i = 0; i < n; i++) {
        const float re = (float)tab[2 * i], im = (float)tab[2 * i + 1];  // the values of tables_f32_m
        tf[4 * i] = re;
        tf[4 * i + 1] = re;
        tf[4 * i + 2] = im;
        tf[4 * i + 3] = im;
    }
}

}  // namespace

void build_tables_f32_paired(int N, std::vector<float> &tab) {
    switch (N / 2) {
        case 64: tables_f32_paired_m<64>(tab); break;
        case 256: tables_f32_paired_m<256>(tab); break;
        case 512: tables_f32_paired_m<512>(tab); break;
        case 1024: tables_f32_paired_m<1024>(tab); break;
        default: tab.clear();
    }
}

void fill_slot_freq(int N, std::vector<int32_t> &sf) {
    switch (N / 2) {
        case 64: slot_freq_m<64>(sf); break;
        case 256: slot_freq_m<256>(sf); break;
        case 512: slot_freq_m<512>(sf); break;
        case 1024: slot_freq_m<1024>(sf); break;
        default: sf.clear();
    }
}

void build_tables_fp64(int N, std::vector<double> &tab) {
    switch (N / 2) {
        case 64: tables_m<64>(tab); break;
        case 256: tables_m<256>(tab); break;
        case 512: tables_m<512>(tab); break;
        case 1024: tables_m<1024>(tab); break;
        default: tab.clear();
    }
}

void build_tables_f32(int N, std::vector<float> &tab) {
    switch (N / 2) {
        case 64: tables_f32_m<64>(tab); break;
        case 256: tables_f32_m<256>(tab); break;
        case 512: tables_f32_m<512>(tab); break;
        case 1024: tables_f32_m<1024>(tab); break;
        default: tab.clear();
    }
}

}  // namespace tfheb
