/*
 * oracle.h -- CPU restatement of the tfhe v1.1 gate-bootstrapping path (TEST INFRASTRUCTURE).
 *
 * This is the parity checker for the GPU engine, nothing else: only tests/, the smoke check
 * and bench.py's CPU-baseline leg load it.  Every product of a torus polynomial by an integer
 * polynomial is EXACT here (negacyclic schoolbook products in 128-bit / wrapping 32-bit integer
 * arithmetic) instead of the reference's truncating FP64 FFT, so this oracle is N-generic (the
 * reference's FFT backends are fixed at N=1024) and defines the error-free result that the GPU's
 * floating-point products are measured against in Torus32 units.
 *
 * Pinned against the reference: tests/test_oracle_golden.py checks every function below against
 * golden vectors produced by the reference library itself (tests/golden/make_golden.py) and,
 * when the reference build is present, against live reference calls on identical inputs.
 *
 * Layouts (all int32, row-major):
 *   LWE sample       [n+1]                 a[0..n-1], b
 *   TLWE sample      [k+1][N]              a[0..k-1], b      (tlwe.h: TLweSample::a, b = a[k])
 *   bootstrapping key[n][kpl][k+1][N]      coefficient-domain TGSW rows, kpl=(k+1)*l, row p=u*l+q
 *   keyswitch key    [k*N][t][base][n+1]   LweKeySwitchKey::ks0_raw order (lwekeyswitch.cpp:3-19)
 */
#ifndef TFHE_B200_ORACLE_H
#define TFHE_B200_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int32_t n;          /* LWE dimension */
    int32_t N;          /* ring degree */
    int32_t k;          /* TLWE mask polynomials */
    int32_t l;          /* gadget decomposition length */
    int32_t Bgbit;      /* log2 of the gadget base */
    int32_t ks_t;       /* keyswitch decomposition length */
    int32_t ks_basebit; /* log2 of the keyswitch base */
} or_params;

/* numeric-functions.cpp:59-65, 71-76 */
int32_t or_modswitch_from(int32_t phase, int32_t Msize);
int32_t or_modswitch_to(int32_t mu, int32_t Msize);

/* tgsw-functions.cpp:297-410 with tgsw.cpp:7-29 (offset, halfBg, maskMod) */
void or_decompose(int32_t N, int32_t l, int32_t Bgbit, const int32_t *poly, int32_t *digits);

/* toruspolynomial-functions.cpp:117-136 and 140-160 */
void or_mul_by_xai_minus_one(int32_t N, int32_t a, const int32_t *in, int32_t *out);
void or_mul_by_xai(int32_t N, int32_t a, const int32_t *in, int32_t *out);

/* Exact negacyclic product d * c in Z[X]/(X^N+1), accumulated in int128 (no reduction).
 * Reduced mod 2^32 it equals torusPolynomialMultNaive_aux (multiplication.cpp:53-65). */
void or_negacyclic_mult_wide(int32_t N, const int32_t *ipoly, const int32_t *tpoly, __int128 *out);
void or_negacyclic_mult(int32_t N, const int32_t *ipoly, const int32_t *tpoly, int32_t *out);

/* One exact external product (tgsw-fft-operations.cpp:89-114 with exact products):
 * acc[(k+1)][N] <- sum_p decomp(acc)_p * bsk_row[p].  If wide != NULL it also receives the
 * int128 sums before reduction ([(k+1)][N]). */
void or_external_product(const or_params *P, const int32_t *bsk_i, int32_t *acc, __int128 *wide);

/* One CMUX step (lwe-bootstrapping-functions-fft.cpp:67-76):
 * acc <- acc + bsk_i [*] ((X^a - 1) acc) */
void or_cmux_step(const or_params *P, const int32_t *bsk_i, int32_t a, int32_t *acc);

/* tfhe_blindRotate_FFT (lwe-bootstrapping-functions-fft.cpp:88-112), exact products. */
void or_blind_rotate(const or_params *P, const int32_t *bsk, const int32_t *bara, int32_t *acc);

/* tLweExtractLweSampleIndex, index 0 (lwe.cpp:41-60): tlwe[(k+1)][N] -> lwe[k*N+1] */
void or_extract(int32_t N, int32_t k, const int32_t *tlwe, int32_t *lwe);

/* tfhe_bootstrap_woKS_FFT (lwe-bootstrapping-functions-fft.cpp:169-200):
 * x[n+1] -> out[k*N+1].  bara_out (optional) receives the n+1 mod-switched values (bara..., barb). */
void or_bootstrap_woks(const or_params *P, const int32_t *bsk, int32_t mu, const int32_t *x,
                       int32_t *out, int32_t *bara_out);

/* lweKeySwitch (lwe-keyswitch-functions.cpp:114-129, 228-238): in[k*N+1] -> out[n+1] */
void or_keyswitch(const or_params *P, const int32_t *ksk, const int32_t *in, int32_t *out);

/* Gate linear combination (boot-gates.cpp:34-319): out[n+1] = (0,const) +- ca +- cb ...
 * gate codes: 0 NAND 1 OR 2 AND 3 XOR 4 XNOR 5 NOR 6 ANDNY 7 ANDYN 8 ORNY 9 ORYN */
void or_gate_prologue(int32_t n, int32_t gate, const int32_t *ca, const int32_t *cb, int32_t *out);

/* Full bootstrapped gate (boot-gates.cpp): binary gates 0..9, MUX = 10 (boot-gates.cpp:329-370),
 * NOT = 11, COPY = 12.  cc is only read by MUX. */
void or_gate(const or_params *P, const int32_t *bsk, const int32_t *ksk, int32_t gate,
             const int32_t *ca, const int32_t *cb, const int32_t *cc, int32_t *out);

/* ---- key generation and encryption (restated from lwe-functions.cpp:20-47,
 *      tlwe-functions.cpp:15-39, tgsw-functions.cpp:118-195, lwe-keyswitch-functions.cpp:163-215,
 *      lwe-bootstrapping-functions.cpp:185-217) with a self-contained seeded generator.
 *      The random stream differs from the reference's std::default_random_engine; the keys are
 *      drawn from the same distributions. ---- */
void or_keygen(const or_params *P, double ks_stdev, double bk_stdev, uint64_t seed,
               int32_t *lwe_key, int32_t *tlwe_key, int32_t *ksk, int32_t *bsk);
void or_lwe_encrypt(int32_t n, const int32_t *key, const int32_t *mus, double stdev, uint64_t seed,
                    int32_t count, int32_t *out);
int32_t or_lwe_phase(int32_t n, const int32_t *key, const int32_t *x);

#ifdef __cplusplus
}
#endif
#endif
