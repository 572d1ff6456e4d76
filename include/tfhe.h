/*
 * tfhe.h -- drop-in replacement for the gate-bootstrapping API of tfhe v1.1, served by
 * libtfhe_b200.so.  A program written against the reference's tfhe.h gate API
 * (tfhe_gate_bootstrapping_functions.h:14-89) compiles against this header unchanged and links
 * with -ltfhe_b200 instead of -ltfhe-spqlios-fma.
 *
 * Struct layouts visible to callers keep the reference's field order and types:
 *   LweParams        lweparams.h:13-16          LweSample   lwesamples.h:9-12
 *   TLweParams       tlwe.h:10-15               LweKey      lwekey.h:10-12
 *   TGswParams       tgsw.h:10-19
 *   TFheGateBootstrappingParameterSet / CloudKeySet / SecretKeySet
 *                    tfhe_gate_bootstrapping_structures.h:9-63
 *   TorusPolynomial  polynomials.h:24-34        TLweSample  tlwe.h:47-51
 *   TGswSample       tgsw.h:55-60               TGswSampleFFT tgsw.h:78-83
 *   LweBootstrappingKey / LweBootstrappingKeyFFT  lwebootstrappingkey.h:10-16, 36-42
 * TGswKey, LweKeySwitchKey and TLweSampleFFT are opaque here.  A cloud keyset's bk->bk is a view of
 * the coefficient-domain key on the host (TGswSample rows whose polynomials point into the key's
 * memory: read them, do not write them); its bkFFT->bkFFT array stands for the FFT-domain key, which
 * lives on the GPU (each TLweSampleFFT is a handle of one key row).
 *
 * Every bootstrapped gate runs on the GPU (no CPU fallback).  The drop-in keeps the reference's
 * FP64 precision by default; tfhe_b200_set_precision selects the split-FP32 form.
 */
#ifndef TFHE_B200_DROPIN_TFHE_H
#define TFHE_B200_DROPIN_TFHE_H

#include <stdint.h>
#include <stdio.h>

#ifdef __cplusplus
#define TFHE_B200_EXPORT extern "C"
#else
#define TFHE_B200_EXPORT
#endif

typedef int32_t Torus32;

typedef struct LweParams {
    const int32_t n;
    const double alpha_min;
    const double alpha_max;
} LweParams;

typedef struct TLweParams {
    const int32_t N;
    const int32_t k;
    const double alpha_min;
    const double alpha_max;
    const LweParams extracted_lweparams;
} TLweParams;

typedef struct TGswParams {
    const int32_t l;
    const int32_t Bgbit;
    const int32_t Bg;
    const int32_t halfBg;
    const uint32_t maskMod;
    const TLweParams *tlwe_params;
    const int32_t kpl;
    Torus32 *h;
    uint32_t offset;
} TGswParams;

typedef struct LweSample {
    Torus32 *a;
    Torus32 b;
    double current_variance;
} LweSample;

typedef struct LweKey {
    const LweParams *params;
    int32_t *key;
} LweKey;

typedef struct TGswKey TGswKey;
typedef struct LweKeySwitchKey LweKeySwitchKey;
typedef struct TLweSampleFFT TLweSampleFFT;

typedef struct TorusPolynomial {
    const int32_t N;
    Torus32 *coefsT;
} TorusPolynomial;

typedef struct TLweSample {
    TorusPolynomial *a;  /* k+1 polynomials: mask, then the body */
    TorusPolynomial *b;  /* alias of a[k] */
    double current_variance;
    const int32_t k;
} TLweSample;

typedef struct TGswSample {
    TLweSample *all_sample;   /* (k+1)*l rows */
    TLweSample **bloc_sample; /* k+1 blocks of l rows */
    const int32_t k;
    const int32_t l;
} TGswSample;

typedef struct TGswSampleFFT {
    TLweSampleFFT *all_samples; /* (k+1)*l row handles */
    TLweSampleFFT **sample;     /* k+1 blocks of l handles */
    const int32_t k;
    const int32_t l;
} TGswSampleFFT;

typedef struct LweBootstrappingKey {
    const LweParams *in_out_params;
    const TGswParams *bk_params;
    const TLweParams *accum_params;
    const LweParams *extract_params;
    TGswSample *bk;      /* n TGSW samples, coefficient domain (host view) */
    LweKeySwitchKey *ks;
} LweBootstrappingKey;

typedef struct LweBootstrappingKeyFFT {
    const LweParams *in_out_params;
    const TGswParams *bk_params;
    const TLweParams *accum_params;
    const LweParams *extract_params;
    const TGswSampleFFT *bkFFT; /* n TGSW samples, FFT domain (on the GPU) */
    const LweKeySwitchKey *ks;
} LweBootstrappingKeyFFT;

typedef struct TFheGateBootstrappingParameterSet {
    const int32_t ks_t;
    const int32_t ks_basebit;
    const LweParams *const in_out_params;
    const TGswParams *const tgsw_params;
} TFheGateBootstrappingParameterSet;

typedef struct TFheGateBootstrappingCloudKeySet {
    const TFheGateBootstrappingParameterSet *const params;
    const LweBootstrappingKey *const bk;
    const LweBootstrappingKeyFFT *const bkFFT;
} TFheGateBootstrappingCloudKeySet;

typedef struct TFheGateBootstrappingSecretKeySet {
    const TFheGateBootstrappingParameterSet *params;
    const LweKey *lwe_key;
    const TGswKey *tgsw_key;
    const TFheGateBootstrappingCloudKeySet cloud;
} TFheGateBootstrappingSecretKeySet;

/* ---- tfhe_gate_bootstrapping_functions.h:14-89 --------------------------------------------- */
/* The gate functions run on the GPU.  Like the reference's, they may be called from several host
 * threads at once on one cloud keyset (each thread with its own results); single-gate calls that
 * arrive together are evaluated as one batch, so throughput grows with the number of calling
 * threads.  A result may alias an operand. */
TFHE_B200_EXPORT TFheGateBootstrappingParameterSet *new_default_gate_bootstrapping_parameters(int32_t minimum_lambda);
TFHE_B200_EXPORT TFheGateBootstrappingSecretKeySet *
new_random_gate_bootstrapping_secret_keyset(const TFheGateBootstrappingParameterSet *params);
TFHE_B200_EXPORT void delete_gate_bootstrapping_parameters(TFheGateBootstrappingParameterSet *params);
TFHE_B200_EXPORT void delete_gate_bootstrapping_secret_keyset(TFheGateBootstrappingSecretKeySet *keyset);
TFHE_B200_EXPORT void delete_gate_bootstrapping_cloud_keyset(TFheGateBootstrappingCloudKeySet *keyset);
TFHE_B200_EXPORT LweSample *new_gate_bootstrapping_ciphertext(const TFheGateBootstrappingParameterSet *params);
TFHE_B200_EXPORT LweSample *new_gate_bootstrapping_ciphertext_array(int32_t nbelems,
                                                                    const TFheGateBootstrappingParameterSet *params);
TFHE_B200_EXPORT void delete_gate_bootstrapping_ciphertext(LweSample *sample);
TFHE_B200_EXPORT void delete_gate_bootstrapping_ciphertext_array(int32_t nbelems, LweSample *samples);
TFHE_B200_EXPORT void bootsSymEncrypt(LweSample *result, int32_t message, const TFheGateBootstrappingSecretKeySet *params);
TFHE_B200_EXPORT int32_t bootsSymDecrypt(const LweSample *sample, const TFheGateBootstrappingSecretKeySet *params);
TFHE_B200_EXPORT void bootsCONSTANT(LweSample *result, int32_t value, const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsNAND(LweSample *result, const LweSample *ca, const LweSample *cb,
                                const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsOR(LweSample *result, const LweSample *ca, const LweSample *cb,
                              const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsAND(LweSample *result, const LweSample *ca, const LweSample *cb,
                               const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsXOR(LweSample *result, const LweSample *ca, const LweSample *cb,
                               const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsXNOR(LweSample *result, const LweSample *ca, const LweSample *cb,
                                const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsNOT(LweSample *result, const LweSample *ca, const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsCOPY(LweSample *result, const LweSample *ca, const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsNOR(LweSample *result, const LweSample *ca, const LweSample *cb,
                               const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsANDNY(LweSample *result, const LweSample *ca, const LweSample *cb,
                                 const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsANDYN(LweSample *result, const LweSample *ca, const LweSample *cb,
                                 const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsORNY(LweSample *result, const LweSample *ca, const LweSample *cb,
                                const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsORYN(LweSample *result, const LweSample *ca, const LweSample *cb,
                                const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsMUX(LweSample *result, const LweSample *a, const LweSample *b, const LweSample *c,
                               const TFheGateBootstrappingCloudKeySet *bk);

/* ---- tfhe.h:34 ------------------------------------------------------------------------------ */
TFHE_B200_EXPORT void tfhe_random_generator_setSeed(uint32_t *values, int32_t size);

/* ---- hot-path internals of tfhe.h:42-45 / lwe-functions.h:79, on the GPU -------------------- */
TFHE_B200_EXPORT void tfhe_bootstrap_FFT(LweSample *result, const LweBootstrappingKeyFFT *bk, Torus32 mu,
                                         const LweSample *x);
TFHE_B200_EXPORT void tfhe_bootstrap_woKS_FFT(LweSample *result, const LweBootstrappingKeyFFT *bk, Torus32 mu,
                                              const LweSample *x);
TFHE_B200_EXPORT Torus32 modSwitchToTorus32(int32_t mu, int32_t Msize);
TFHE_B200_EXPORT int32_t modSwitchFromTorus32(Torus32 phase, int32_t Msize);
TFHE_B200_EXPORT Torus32 lwePhase(const LweSample *sample, const LweKey *key);

/* ---- batched extensions (no reference counterpart: the reference evaluates one gate per call) -
 * results[i] = gate(a[i], b[i] (, c[i])) for i < count, over arrays from
 * new_gate_bootstrapping_ciphertext_array; one GPU launch sequence per call.
 * gate codes as in tfhe_b200.h (0 NAND ... 10 MUX, 11 NOT, 12 COPY). */
TFHE_B200_EXPORT void bootsGATE_batch(int32_t gate, LweSample *results, const LweSample *a, const LweSample *b,
                                      const LweSample *c, int32_t count, const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsNAND_batch(LweSample *results, const LweSample *a, const LweSample *b, int32_t count,
                                      const TFheGateBootstrappingCloudKeySet *bk);
TFHE_B200_EXPORT void bootsMUX_batch(LweSample *results, const LweSample *a, const LweSample *b, const LweSample *c,
                                     int32_t count, const TFheGateBootstrappingCloudKeySet *bk);

/* ---- tfhe.h:36-43, tgsw_functions.h:40-46, lwe-functions.h:79: blind rotation, external product
 * and keyswitch on single samples, on the GPU.
 *   tfhe_blindRotate_FFT(accum, bk, bara, n, params): accum *= X^{sum bara_i s_i} over the n TGSW
 *     samples bk[0..n-1]; bk must point into a keyset's bkFFT->bkFFT array (any offset).
 *   tfhe_blindRotateAndExtract_FFT: the same from the test vector (0, X^{2N-barb} v), then the sample
 *     extraction at index 0 into result (dimension kN).
 *   tfhe_blindRotate / tfhe_blindRotateAndExtract: the same on coefficient-domain TGSW samples: a
 *     keyset's bk->bk rows run on that key's device key; other TGSW samples are moved to the GPU and
 *     transformed on every call (each call then allocates device memory).
 *   tGswExternProduct(result, a, b, params): result = a (x) b; tGswExternMulToTLwe(accum, sample,
 *     params): accum = sample (x) accum.
 *   lweKeySwitch(result, ks, sample): ks must be a keyset's bk->ks or bkFFT->ks.
 * The products use the FP64 FFT by default (split-FP32 after tfhe_b200_set_precision(1)); the
 * reference's coefficient-domain functions compute them exactly, so their results may differ from
 * it by a unit in rare coefficients.  Variances follow the reference's bookkeeping: the rotations
 * keep accum's, tGswExternProduct and tGswExternMulToTLwe add ||digits||^2 times each TGSW row's
 * variance (plus b's), lweKeySwitch and every keyswitched bootstrap sum the keyswitching-key rows'
 * variances over the non-zero digits, and tfhe_bootstrap_woKS(_FFT) and the extractions leave the
 * result's variance as it was. */
TFHE_B200_EXPORT void tfhe_blindRotate_FFT(TLweSample *accum, const TGswSampleFFT *bk, const int32_t *bara,
                                           const int32_t n, const TGswParams *bk_params);
TFHE_B200_EXPORT void tfhe_blindRotateAndExtract_FFT(LweSample *result, const TorusPolynomial *v,
                                                     const TGswSampleFFT *bk, const int32_t barb,
                                                     const int32_t *bara, const int32_t n,
                                                     const TGswParams *bk_params);
TFHE_B200_EXPORT void tfhe_blindRotate(TLweSample *accum, const TGswSample *bk, const int32_t *bara, const int32_t n,
                                       const TGswParams *bk_params);
TFHE_B200_EXPORT void tfhe_blindRotateAndExtract(LweSample *result, const TorusPolynomial *v, const TGswSample *bk,
                                                 const int32_t barb, const int32_t *bara, const int32_t n,
                                                 const TGswParams *bk_params);
TFHE_B200_EXPORT void tGswExternProduct(TLweSample *result, const TGswSample *a, const TLweSample *b,
                                        const TGswParams *params);
TFHE_B200_EXPORT void tGswExternMulToTLwe(TLweSample *accum, const TGswSample *sample, const TGswParams *params);
TFHE_B200_EXPORT void lweKeySwitch(LweSample *result, const LweKeySwitchKey *ks, const LweSample *sample);

/* ---- polynomials.h:97-103, tlwe.h:222-235, lwesamples.h:70-83: allocation of the samples above --- */
TFHE_B200_EXPORT TorusPolynomial *new_TorusPolynomial(const int32_t N);
TFHE_B200_EXPORT TorusPolynomial *new_TorusPolynomial_array(int32_t nbelts, const int32_t N);
TFHE_B200_EXPORT void delete_TorusPolynomial(TorusPolynomial *obj);
TFHE_B200_EXPORT void delete_TorusPolynomial_array(int32_t nbelts, TorusPolynomial *obj);
TFHE_B200_EXPORT TLweSample *new_TLweSample(const TLweParams *params);
TFHE_B200_EXPORT TLweSample *new_TLweSample_array(int32_t nbelts, const TLweParams *params);
TFHE_B200_EXPORT void delete_TLweSample(TLweSample *obj);
TFHE_B200_EXPORT void delete_TLweSample_array(int32_t nbelts, TLweSample *obj);
TFHE_B200_EXPORT LweSample *new_LweSample(const LweParams *params);
TFHE_B200_EXPORT LweSample *new_LweSample_array(int32_t nbelts, const LweParams *params);
TFHE_B200_EXPORT void delete_LweSample(LweSample *obj);
TFHE_B200_EXPORT void delete_LweSample_array(int32_t nbelts, LweSample *obj);

/* ---- tfhe.h:38-39: coefficient-domain bootstrap (same GPU path as the _FFT forms) ------------ */
TFHE_B200_EXPORT void tfhe_bootstrap(LweSample *result, const LweBootstrappingKey *bk, Torus32 mu, const LweSample *x);
TFHE_B200_EXPORT void tfhe_bootstrap_woKS(LweSample *result, const LweBootstrappingKey *bk, Torus32 mu,
                                          const LweSample *x);

/* ---- lwe-functions.h:25-68 and numeric-functions.h (approxPhase): host-side LWE helpers ------- */
TFHE_B200_EXPORT void lweSymEncrypt(LweSample *result, Torus32 message, double alpha, const LweKey *key);
TFHE_B200_EXPORT void lweSymEncryptWithExternalNoise(LweSample *result, Torus32 message, double noise, double alpha,
                                                     const LweKey *key);
TFHE_B200_EXPORT Torus32 lweSymDecrypt(const LweSample *sample, const LweKey *key, const int32_t Msize);
TFHE_B200_EXPORT Torus32 approxPhase(Torus32 phase, int32_t Msize);
TFHE_B200_EXPORT void lweClear(LweSample *result, const LweParams *params);
TFHE_B200_EXPORT void lweCopy(LweSample *result, const LweSample *sample, const LweParams *params);
TFHE_B200_EXPORT void lweNegate(LweSample *result, const LweSample *sample, const LweParams *params);
TFHE_B200_EXPORT void lweNoiselessTrivial(LweSample *result, Torus32 mu, const LweParams *params);
TFHE_B200_EXPORT void lweAddTo(LweSample *result, const LweSample *sample, const LweParams *params);
TFHE_B200_EXPORT void lweSubTo(LweSample *result, const LweSample *sample, const LweParams *params);
TFHE_B200_EXPORT void lweAddMulTo(LweSample *result, int32_t p, const LweSample *sample, const LweParams *params);
TFHE_B200_EXPORT void lweSubMulTo(LweSample *result, int32_t p, const LweSample *sample, const LweParams *params);

/* ---- tfhe_io.h: files in the reference's format (tfhe_io.cpp:90-136, 1010-1220) -------------
 * Same layout byte for byte, so key sets and ciphertexts move between this library and tfhe. */
TFHE_B200_EXPORT void export_lweSample_toFile(FILE *F, const LweSample *lwesample, const LweParams *params);
TFHE_B200_EXPORT void import_lweSample_fromFile(FILE *F, LweSample *lwesample, const LweParams *params);
TFHE_B200_EXPORT void export_gate_bootstrapping_ciphertext_toFile(FILE *F, const LweSample *sample,
                                                                  const TFheGateBootstrappingParameterSet *params);
TFHE_B200_EXPORT void import_gate_bootstrapping_ciphertext_fromFile(FILE *F, LweSample *sample,
                                                                    const TFheGateBootstrappingParameterSet *params);
TFHE_B200_EXPORT void export_tfheGateBootstrappingParameterSet_toFile(FILE *F,
                                                                      const TFheGateBootstrappingParameterSet *params);
TFHE_B200_EXPORT TFheGateBootstrappingParameterSet *new_tfheGateBootstrappingParameterSet_fromFile(FILE *F);
TFHE_B200_EXPORT void export_tfheGateBootstrappingCloudKeySet_toFile(FILE *F,
                                                                     const TFheGateBootstrappingCloudKeySet *keyset);
TFHE_B200_EXPORT TFheGateBootstrappingCloudKeySet *new_tfheGateBootstrappingCloudKeySet_fromFile(FILE *F);
TFHE_B200_EXPORT void export_tfheGateBootstrappingSecretKeySet_toFile(FILE *F,
                                                                      const TFheGateBootstrappingSecretKeySet *keyset);
TFHE_B200_EXPORT TFheGateBootstrappingSecretKeySet *new_tfheGateBootstrappingSecretKeySet_fromFile(FILE *F);

/* 0 = FP64 (default), 1 = split FP32.  Applies to subsequent gate calls of this process. */
TFHE_B200_EXPORT void tfhe_b200_set_precision(int32_t precision);

#endif
