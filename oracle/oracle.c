/*
 * oracle.c -- CPU restatement of the tfhe v1.1 gate-bootstrapping path (TEST INFRASTRUCTURE).
 * See oracle.h for the contract.  Only tests/, the smoke check and bench.py's CPU-baseline leg
 * load this code; the GPU engine never links it.
 *
 * Citations are to the reference sources (paths relative to the tfhe repository root).
 */
#include "oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ------------------------------------------------------------------------------------------ */
/* numerics: src/libtfhe/numeric-functions.cpp                                                 */
/* ------------------------------------------------------------------------------------------ */

/* numeric-functions.cpp:59-65: round(phase * Msize) mod Msize, computed on 64 bits. */
int32_t or_modswitch_from(int32_t phase, int32_t Msize) {
    const uint64_t interv = ((UINT64_C(1) << 63) / (uint64_t)Msize) * 2;
    const uint64_t half = interv / 2;
    const uint64_t phase64 = ((uint64_t)(uint32_t)phase << 32) + half;
    return (int32_t)(phase64 / interv);
}

/* numeric-functions.cpp:71-76: mu / Msize as a Torus32. */
int32_t or_modswitch_to(int32_t mu, int32_t Msize) {
    const uint64_t interv = ((UINT64_C(1) << 63) / (uint64_t)Msize) * 2;
    const uint64_t phase64 = (uint64_t)(int64_t)mu * interv;
    return (int32_t)(uint32_t)(phase64 >> 32);
}

/* numeric-functions.cpp:33-35: fractional part of d as a Torus32 (truncating). */
static int32_t or_dtot32(double d) {
    const double frac = d - (double)(int64_t)d;
    return (int32_t)(uint32_t)(uint64_t)(int64_t)(frac * 4294967296.0);
}

/* ------------------------------------------------------------------------------------------ */
/* gadget decomposition: tgsw-functions.cpp:297-410, constants from tgsw.cpp:7-29              */
/* ------------------------------------------------------------------------------------------ */

static uint32_t gadget_offset(int32_t l, int32_t Bgbit) {
    uint32_t sum = 0;
    for (int32_t i = 0; i < l; i++) sum += (uint32_t)1 << (32 - (i + 1) * Bgbit);
    return sum * (uint32_t)(1 << (Bgbit - 1));
}

void or_decompose(int32_t N, int32_t l, int32_t Bgbit, const int32_t *poly, int32_t *digits) {
    const uint32_t offset = gadget_offset(l, Bgbit);
    const uint32_t mask = ((uint32_t)1 << Bgbit) - 1;
    const int32_t halfBg = 1 << (Bgbit - 1);
    for (int32_t p = 0; p < l; p++) {
        const int32_t shift = 32 - (p + 1) * Bgbit;
        for (int32_t j = 0; j < N; j++) {
            const uint32_t v = (uint32_t)poly[j] + offset;
            digits[p * N + j] = (int32_t)((v >> shift) & mask) - halfBg;
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* rotations: toruspolynomial-functions.cpp:117-160                                            */
/* ------------------------------------------------------------------------------------------ */

/* out = X^a * in in Z[X]/(X^N+1), 0 <= a < 2N */
void or_mul_by_xai(int32_t N, int32_t a, const int32_t *in, int32_t *out) {
    for (int32_t i = 0; i < N; i++) {
        /* coefficient i of X^a*in is +-in[(i-a) mod N], negated once per wrap past X^N */
        int32_t src = i - a;
        uint32_t neg = 0;
        while (src < 0) { src += N; neg ^= 1u; }
        const uint32_t v = (uint32_t)in[src];
        out[i] = (int32_t)(neg ? (0u - v) : v);
    }
}

/* out = (X^a - 1) * in */
void or_mul_by_xai_minus_one(int32_t N, int32_t a, const int32_t *in, int32_t *out) {
    for (int32_t i = 0; i < N; i++) {
        int32_t src = i - a;
        uint32_t neg = 0;
        while (src < 0) { src += N; neg ^= 1u; }
        const uint32_t v = (uint32_t)in[src];
        out[i] = (int32_t)((neg ? (0u - v) : v) - (uint32_t)in[i]);
    }
}

/* ------------------------------------------------------------------------------------------ */
/* exact negacyclic products (semantics of multiplication.cpp:53-65)                           */
/* ------------------------------------------------------------------------------------------ */

void or_negacyclic_mult_wide(int32_t N, const int32_t *ipoly, const int32_t *tpoly, __int128 *out) {
    for (int32_t i = 0; i < N; i++) out[i] = 0;
    for (int32_t j = 0; j < N; j++) {
        const __int128 d = ipoly[j];
        if (d == 0) continue;
        for (int32_t i = 0; i < N - j; i++) out[i + j] += d * (__int128)tpoly[i];
        for (int32_t i = N - j; i < N; i++) out[i + j - N] -= d * (__int128)tpoly[i];
    }
}

/* Same product reduced mod 2^32, in wrapping 32-bit arithmetic (exact mod 2^32). */
static void negacyclic_addmul_u32(int32_t N, const int32_t *ipoly, const int32_t *tpoly, uint32_t *acc) {
    for (int32_t j = 0; j < N; j++) {
        const uint32_t d = (uint32_t)ipoly[j];
        if (d == 0) continue;
        uint32_t *hi = acc + j;
        const uint32_t *t = (const uint32_t *)tpoly;
        for (int32_t i = 0; i < N - j; i++) hi[i] += d * t[i];
        uint32_t *lo = acc + j - N;
        for (int32_t i = N - j; i < N; i++) lo[i] -= d * t[i];
    }
}

void or_negacyclic_mult(int32_t N, const int32_t *ipoly, const int32_t *tpoly, int32_t *out) {
    memset(out, 0, sizeof(int32_t) * (size_t)N);
    negacyclic_addmul_u32(N, ipoly, tpoly, (uint32_t *)out);
}

/* ------------------------------------------------------------------------------------------ */
/* external product, CMUX, blind rotation: tgsw-fft-operations.cpp:89-114,                     */
/* lwe-bootstrapping-functions-fft.cpp:67-156                                                   */
/* ------------------------------------------------------------------------------------------ */

void or_external_product(const or_params *P, const int32_t *bsk_i, int32_t *acc, __int128 *wide) {
    const int32_t N = P->N, k = P->k, l = P->l, kpl = (P->k + 1) * P->l;
    int32_t *dec = (int32_t *)malloc(sizeof(int32_t) * (size_t)kpl * N);
    uint32_t *res = (uint32_t *)calloc((size_t)(k + 1) * N, sizeof(uint32_t));
    /* rows p = u*l + q: digit q of polynomial u (tgsw-fft-operations.cpp:100-101) */
    for (int32_t u = 0; u <= k; u++) or_decompose(N, l, P->Bgbit, acc + u * N, dec + u * l * N);
    for (int32_t p = 0; p < kpl; p++)
        for (int32_t v = 0; v <= k; v++)
            negacyclic_addmul_u32(N, dec + p * N, bsk_i + ((size_t)p * (k + 1) + v) * N, res + v * N);
    if (wide) {
        __int128 *tmp = (__int128 *)malloc(sizeof(__int128) * (size_t)N);
        for (int32_t i = 0; i < (k + 1) * N; i++) wide[i] = 0;
        for (int32_t p = 0; p < kpl; p++)
            for (int32_t v = 0; v <= k; v++) {
                or_negacyclic_mult_wide(N, dec + p * N, bsk_i + ((size_t)p * (k + 1) + v) * N, tmp);
                for (int32_t i = 0; i < N; i++) wide[v * N + i] += tmp[i];
            }
        free(tmp);
    }
    memcpy(acc, res, sizeof(int32_t) * (size_t)(k + 1) * N);
    free(res);
    free(dec);
}

void or_cmux_step(const or_params *P, const int32_t *bsk_i, int32_t a, int32_t *acc) {
    const int32_t N = P->N, k = P->k;
    int32_t *tmp = (int32_t *)malloc(sizeof(int32_t) * (size_t)(k + 1) * N);
    for (int32_t u = 0; u <= k; u++) or_mul_by_xai_minus_one(N, a, acc + u * N, tmp + u * N);
    or_external_product(P, bsk_i, tmp, NULL);
    for (int32_t i = 0; i < (k + 1) * N; i++) acc[i] = (int32_t)((uint32_t)acc[i] + (uint32_t)tmp[i]);
    free(tmp);
}

void or_blind_rotate(const or_params *P, const int32_t *bsk, const int32_t *bara, int32_t *acc) {
    const size_t row = (size_t)(P->k + 1) * P->l * (P->k + 1) * P->N;
    for (int32_t i = 0; i < P->n; i++) {
        if (bara[i] == 0) continue; /* lwe-bootstrapping-functions-fft.cpp:101 */
        or_cmux_step(P, bsk + (size_t)i * row, bara[i], acc);
    }
}

/* lwe.cpp:41-53 with index 0 */
void or_extract(int32_t N, int32_t k, const int32_t *tlwe, int32_t *lwe) {
    for (int32_t i = 0; i < k; i++) {
        lwe[i * N] = tlwe[i * N];
        for (int32_t j = 1; j < N; j++) lwe[i * N + j] = (int32_t)(0u - (uint32_t)tlwe[i * N + N - j]);
    }
    lwe[k * N] = tlwe[k * N];
}

void or_bootstrap_woks(const or_params *P, const int32_t *bsk, int32_t mu, const int32_t *x,
                       int32_t *out, int32_t *bara_out) {
    const int32_t N = P->N, k = P->k, n = P->n, Nx2 = 2 * P->N;
    int32_t *bara = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    int32_t *testvect = (int32_t *)malloc(sizeof(int32_t) * (size_t)N);
    int32_t *acc = (int32_t *)calloc((size_t)(k + 1) * N, sizeof(int32_t));
    const int32_t barb = or_modswitch_from(x[n], Nx2);
    for (int32_t i = 0; i < n; i++) bara[i] = or_modswitch_from(x[i], Nx2);
    if (bara_out) {
        memcpy(bara_out, bara, sizeof(int32_t) * (size_t)n);
        bara_out[n] = barb;
    }
    for (int32_t i = 0; i < N; i++) testvect[i] = mu;
    /* acc = (0, X^{2N-barb} * v)  (lwe-bootstrapping-functions-fft.cpp:142-145) */
    if (barb != 0) or_mul_by_xai(N, Nx2 - barb, testvect, acc + k * N);
    else memcpy(acc + k * N, testvect, sizeof(int32_t) * (size_t)N);
    or_blind_rotate(P, bsk, bara, acc);
    or_extract(N, k, acc, out);
    free(acc);
    free(testvect);
    free(bara);
}

/* ------------------------------------------------------------------------------------------ */
/* keyswitch: lwe-keyswitch-functions.cpp:114-129, 228-238                                     */
/* ------------------------------------------------------------------------------------------ */

void or_keyswitch(const or_params *P, const int32_t *ksk, const int32_t *in, int32_t *out) {
    const int32_t n = P->n, kN = P->k * P->N, t = P->ks_t, basebit = P->ks_basebit;
    const int32_t base = 1 << basebit;
    const uint32_t prec_offset = (uint32_t)1 << (32 - (1 + basebit * t));
    const uint32_t mask = (uint32_t)base - 1;
    uint32_t *r = (uint32_t *)out;
    for (int32_t i = 0; i < n; i++) r[i] = 0;
    r[n] = (uint32_t)in[kN];
    for (int32_t i = 0; i < kN; i++) {
        const uint32_t aibar = (uint32_t)in[i] + prec_offset;
        for (int32_t j = 0; j < t; j++) {
            const uint32_t aij = (aibar >> (32 - (j + 1) * basebit)) & mask;
            if (aij == 0) continue;
            const uint32_t *row = (const uint32_t *)ksk + (((size_t)i * t + j) * base + aij) * (size_t)(n + 1);
            for (int32_t c = 0; c <= n; c++) r[c] -= row[c];
        }
    }
}

/* ------------------------------------------------------------------------------------------ */
/* gates: boot-gates.cpp                                                                       */
/* ------------------------------------------------------------------------------------------ */

/* Linear combination (0,c) + sa*ca + sb*cb for the ten binary gates (boot-gates.cpp:34-319). */
void or_gate_prologue(int32_t n, int32_t gate, const int32_t *ca, const int32_t *cb, int32_t *out) {
    static const int32_t cnum[10] = {1, 1, -1, 1, -1, -1, -1, -1, 1, 1};
    static const int32_t cden[10] = {8, 8, 8, 4, 4, 8, 8, 8, 8, 8};
    static const int32_t sa[10] = {-1, 1, 1, 2, -2, -1, -1, 1, -1, 1};
    static const int32_t sb[10] = {-1, 1, 1, 2, -2, -1, 1, -1, 1, -1};
    const uint32_t c = (uint32_t)or_modswitch_to(cnum[gate], cden[gate]);
    for (int32_t i = 0; i <= n; i++)
        out[i] = (int32_t)((i == n ? c : 0u) + (uint32_t)sa[gate] * (uint32_t)ca[i] +
                           (uint32_t)sb[gate] * (uint32_t)cb[i]);
}

void or_gate(const or_params *P, const int32_t *bsk, const int32_t *ksk, int32_t gate,
             const int32_t *ca, const int32_t *cb, const int32_t *cc, int32_t *out) {
    const int32_t n = P->n, kN = P->k * P->N;
    const int32_t MU = or_modswitch_to(1, 8);
    if (gate == 11) { /* NOT: boot-gates.cpp:164-167 */
        for (int32_t i = 0; i <= n; i++) out[i] = (int32_t)(0u - (uint32_t)ca[i]);
        return;
    }
    if (gate == 12) { /* COPY */
        memcpy(out, ca, sizeof(int32_t) * (size_t)(n + 1));
        return;
    }
    int32_t *tmp = (int32_t *)malloc(sizeof(int32_t) * (size_t)(n + 1));
    int32_t *u1 = (int32_t *)malloc(sizeof(int32_t) * (size_t)(kN + 1));
    if (gate == 10) { /* MUX: boot-gates.cpp:329-370 */
        int32_t *u2 = (int32_t *)malloc(sizeof(int32_t) * (size_t)(kN + 1));
        or_gate_prologue(n, 2, ca, cb, tmp);           /* (0,-1/8) + a + b */
        or_bootstrap_woks(P, bsk, MU, tmp, u1, NULL);
        or_gate_prologue(n, 6, ca, cc, tmp);           /* (0,-1/8) - a + c */
        or_bootstrap_woks(P, bsk, MU, tmp, u2, NULL);
        for (int32_t i = 0; i <= kN; i++)
            u1[i] = (int32_t)((uint32_t)u1[i] + (uint32_t)u2[i] + (i == kN ? (uint32_t)MU : 0u));
        or_keyswitch(P, ksk, u1, out);
        free(u2);
    } else {
        or_gate_prologue(n, gate, ca, cb, tmp);
        or_bootstrap_woks(P, bsk, MU, tmp, u1, NULL);
        or_keyswitch(P, ksk, u1, out);
    }
    free(u1);
    free(tmp);
}

/* ------------------------------------------------------------------------------------------ */
/* key generation and encryption                                                               */
/* ------------------------------------------------------------------------------------------ */

typedef struct { uint64_t s[4]; int have_spare; double spare; } or_rng;

static uint64_t splitmix64(uint64_t *x) {
    uint64_t z = (*x += UINT64_C(0x9E3779B97F4A7C15));
    z = (z ^ (z >> 30)) * UINT64_C(0xBF58476D1CE4E5B9);
    z = (z ^ (z >> 27)) * UINT64_C(0x94D049BB133111EB);
    return z ^ (z >> 31);
}

static void rng_init(or_rng *r, uint64_t seed) {
    for (int i = 0; i < 4; i++) r->s[i] = splitmix64(&seed);
    r->have_spare = 0;
}

static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }

/* xoshiro256** */
static uint64_t rng_next(or_rng *r) {
    uint64_t *s = r->s;
    const uint64_t result = rotl(s[1] * 5, 7) * 9;
    const uint64_t t = s[1] << 17;
    s[2] ^= s[0]; s[3] ^= s[1]; s[1] ^= s[2]; s[0] ^= s[3];
    s[2] ^= t; s[3] = rotl(s[3], 45);
    return result;
}

static int32_t rng_torus(or_rng *r) { return (int32_t)(uint32_t)(rng_next(r) >> 32); }
static int32_t rng_bit(or_rng *r) { return (int32_t)(rng_next(r) >> 63); }

/* standard normal by the Marsaglia polar method */
static double rng_normal(or_rng *r) {
    if (r->have_spare) { r->have_spare = 0; return r->spare; }
    double u, v, s;
    do {
        u = (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
        v = (double)(rng_next(r) >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
        s = u * u + v * v;
    } while (s >= 1.0 || s == 0.0);
    const double m = sqrt(-2.0 * log(s) / s);
    r->spare = v * m;
    r->have_spare = 1;
    return u * m;
}

/* lweSymEncryptWithExternalNoise (lwe-functions.cpp:52-63) */
static void lwe_encrypt_noise(or_rng *r, int32_t n, const int32_t *key, int32_t mu, double noise, int32_t *out) {
    uint32_t b = (uint32_t)mu + (uint32_t)or_dtot32(noise);
    for (int32_t i = 0; i < n; i++) {
        out[i] = rng_torus(r);
        b += (uint32_t)out[i] * (uint32_t)key[i];
    }
    out[n] = (int32_t)b;
}

void or_keygen(const or_params *P, double ks_stdev, double bk_stdev, uint64_t seed,
               int32_t *lwe_key, int32_t *tlwe_key, int32_t *ksk, int32_t *bsk) {
    const int32_t n = P->n, N = P->N, k = P->k, l = P->l, kN = P->k * P->N;
    const int32_t t = P->ks_t, basebit = P->ks_basebit, base = 1 << basebit, kpl = (k + 1) * l;
    or_rng r;
    rng_init(&r, seed);
    for (int32_t i = 0; i < n; i++) lwe_key[i] = rng_bit(&r);        /* lwe-functions.cpp:20-26 */
    for (int32_t i = 0; i < kN; i++) tlwe_key[i] = rng_bit(&r);      /* tlwe-functions.cpp:15-23 */

    /* keyswitch key: centred Gaussian noises, h=0 rows trivial zero (lwe-keyswitch-functions.cpp:163-215) */
    const int64_t sizeks = (int64_t)kN * t * (base - 1);
    double *noise = (double *)malloc(sizeof(double) * (size_t)sizeks);
    double mean = 0;
    for (int64_t i = 0; i < sizeks; i++) { noise[i] = rng_normal(&r) * ks_stdev; mean += noise[i]; }
    mean /= (double)sizeks;
    for (int64_t i = 0; i < sizeks; i++) noise[i] -= mean;
    int64_t idx = 0;
    for (int32_t i = 0; i < kN; i++)
        for (int32_t j = 0; j < t; j++) {
            int32_t *row0 = ksk + (((size_t)i * t + j) * base) * (size_t)(n + 1);
            memset(row0, 0, sizeof(int32_t) * (size_t)(n + 1));
            for (int32_t h = 1; h < base; h++) {
                const int32_t mess = (int32_t)((uint32_t)(tlwe_key[i] * h) << (32 - (j + 1) * basebit));
                lwe_encrypt_noise(&r, n, lwe_key, mess, noise[idx++], row0 + (size_t)h * (n + 1));
            }
        }
    free(noise);

    /* bootstrapping key: tGswSymEncryptInt(s_i) per input coefficient (lwe-bootstrapping-functions.cpp:210-214) */
    int32_t *prod = (int32_t *)malloc(sizeof(int32_t) * (size_t)N);
    for (int32_t i = 0; i < n; i++)
        for (int32_t p = 0; p < kpl; p++) {
            int32_t *row = bsk + ((size_t)i * kpl + p) * (size_t)(k + 1) * N;
            int32_t *b = row + (size_t)k * N;
            /* tLweSymEncryptZero (tlwe-functions.cpp:26-39), exact products */
            for (int32_t j = 0; j < N; j++) b[j] = or_dtot32(rng_normal(&r) * bk_stdev);
            for (int32_t u = 0; u < k; u++) {
                int32_t *a = row + (size_t)u * N;
                for (int32_t j = 0; j < N; j++) a[j] = rng_torus(&r);
                or_negacyclic_mult(N, tlwe_key + u * N, a, prod);
                for (int32_t j = 0; j < N; j++) b[j] = (int32_t)((uint32_t)b[j] + (uint32_t)prod[j]);
            }
            /* tGswAddMuIntH (tgsw-functions.cpp:111-122): row (bloc,q) gets mu*h_q on component bloc */
            const int32_t bloc = p / l, q = p % l;
            const uint32_t hq = (uint32_t)1 << (32 - (q + 1) * P->Bgbit);
            row[(size_t)bloc * N] = (int32_t)((uint32_t)row[(size_t)bloc * N] + (uint32_t)lwe_key[i] * hq);
        }
    free(prod);
}

void or_lwe_encrypt(int32_t n, const int32_t *key, const int32_t *mus, double stdev, uint64_t seed,
                    int32_t count, int32_t *out) {
    or_rng r;
    rng_init(&r, seed);
    for (int32_t g = 0; g < count; g++)
        lwe_encrypt_noise(&r, n, key, mus[g], rng_normal(&r) * stdev, out + (size_t)g * (n + 1));
}

int32_t or_lwe_phase(int32_t n, const int32_t *key, const int32_t *x) {
    uint32_t axs = 0;
    for (int32_t i = 0; i < n; i++) axs += (uint32_t)x[i] * (uint32_t)key[i];
    return (int32_t)((uint32_t)x[n] - axs);
}
