/*
 * tfhe_b200.h -- native C ABI of the B200 gate-bootstrapping engine (libtfhe_b200.so).
 *
 * Plain C: pointers, sizes and status codes only.  Ciphertexts are raw int32 arrays:
 *   LWE ciphertext      [n+1]              a[0..n-1], b          (lwesamples.h:9-20: LweSample a, b)
 *   batch of ciphertexts[count][n+1]       row-major
 *   extracted sample    [k*N+1]            dimension of the extracted key (tlwe.h:15 extracted_lweparams)
 * Gate codes follow boot-gates.cpp: 0 NAND 1 OR 2 AND 3 XOR 4 XNOR 5 NOR 6 ANDNY 7 ANDYN 8 ORNY
 * 9 ORYN 10 MUX 11 NOT 12 COPY.
 *
 * Each entry point below names the reference interface it replaces (file:line in tfhe v1.1).
 * The reference-compatible drop-in (same struct layouts and symbols as tfhe_gate_bootstrapping_
 * functions.h) is declared in tfhe.h and implemented on top of this ABI.
 */
#ifndef TFHE_B200_H
#define TFHE_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    TFHEB_OK = 0,
    TFHEB_ERR_INVALID = 1,     /* bad argument or size */
    TFHEB_ERR_CUDA = 2,        /* CUDA runtime error (message in tfheb_last_error) */
    TFHEB_ERR_NOMEM = 3,       /* device or host allocation failed */
    TFHEB_ERR_UNSUPPORTED = 4, /* parameter set without a compiled kernel */
    TFHEB_ERR_TIMEOUT = 5,     /* a bounded device-side wait expired */
    TFHEB_ERR_NO_DEVICE = 6    /* no CUDA device visible */
} tfheb_status;

typedef enum {
    TFHEB_FP64 = 0,       /* plain form: FP64 negacyclic FFT (the reference's precision) */
    TFHEB_SPLIT_FP32 = 1  /* bootstrapping key split in two integer limbs, FP32 FFTs, exact recombination */
} tfheb_precision;

enum {
    TFHEB_NAND = 0, TFHEB_OR = 1, TFHEB_AND = 2, TFHEB_XOR = 3, TFHEB_XNOR = 4, TFHEB_NOR = 5,
    TFHEB_ANDNY = 6, TFHEB_ANDYN = 7, TFHEB_ORNY = 8, TFHEB_ORYN = 9, TFHEB_MUX = 10, TFHEB_NOT = 11,
    TFHEB_COPY = 12
};

/* Gate-bootstrapping parameter set (tfhe_gate_bootstrapping_structures.h:9-24 with the LweParams,
 * TLweParams and TGswParams it points to, flattened). */
typedef struct {
    int32_t n;          /* LWE dimension (lweparams.h:13-16) */
    int32_t N;          /* ring degree (tlwe.h:10-15) */
    int32_t k;          /* TLWE mask polynomials */
    int32_t l;          /* gadget decomposition length (tgsw.h:10-19) */
    int32_t Bgbit;      /* log2 of the gadget base */
    int32_t ks_t;       /* keyswitch length */
    int32_t ks_basebit; /* keyswitch log2 base */
    double ks_stdev;    /* LWE / keyswitch noise stdev (alpha_min of the LWE params) */
    double bk_stdev;    /* bootstrapping-key noise stdev (alpha_min of the TLWE params) */
} tfheb_params;

typedef struct tfheb_secret_key tfheb_secret_key;
typedef struct tfheb_cloud_key tfheb_cloud_key;

/* Last error message of the calling thread ("" if none). */
const char *tfheb_last_error(void);

/* Number of kernels this library launched on the calling process so far (all keys). */
int64_t tfheb_kernel_launches(void);

/* Replaces new_default_gate_bootstrapping_parameters (tfhe_gate_bootstrapping.cpp:77-89):
 * lambda <= 80 -> the 80-bit set (:23-48), 80 < lambda <= 128 -> the 128-bit default (:51-75). */
tfheb_status tfheb_default_params(int32_t lambda, tfheb_params *out);

/* The larger-ring set n=800, N=2048, l=3, Bgbit=8 (no reference counterpart: the reference's FFT
 * backends are fixed at N=1024, fft_processor_spqlios.cpp:123). */
tfheb_status tfheb_large_params(tfheb_params *out);

/* Replaces new_random_gate_bootstrapping_secret_keyset (tfhe_gate_bootstrapping.cpp:97-108):
 * secret keys, keyswitching key and coefficient-domain bootstrapping key, from a seed. */
tfheb_status tfheb_keygen(const tfheb_params *p, uint64_t seed, tfheb_secret_key **sk, tfheb_cloud_key **ck);

/* Import keys generated elsewhere (e.g. by the reference library), raw layouts:
 *   bsk [n][(k+1)*l][k+1][N] coefficient-domain TGSW rows (tgsw.h:55-60 all_sample order)
 *   ksk [k*N][ks_t][2^ks_basebit][n+1] (lwekeyswitch.h:11-28 ks0_raw order); may be NULL for a key
 *       that only serves blind rotations and external products (keyswitches and gates then return
 *       TFHEB_ERR_INVALID, and the key cannot be saved)
 *   lwe_key [n], tlwe_key [k][N]. */
tfheb_status tfheb_cloud_key_import(const tfheb_params *p, const int32_t *bsk, const int32_t *ksk,
                                    tfheb_cloud_key **ck);
tfheb_status tfheb_secret_key_import(const tfheb_params *p, const int32_t *lwe_key, const int32_t *tlwe_key,
                                     tfheb_secret_key **sk);
tfheb_status tfheb_secret_key_export(const tfheb_secret_key *sk, int32_t *lwe_key, int32_t *tlwe_key);
tfheb_status tfheb_cloud_key_export(const tfheb_cloud_key *ck, int32_t *bsk, int32_t *ksk);
tfheb_status tfheb_cloud_key_params(const tfheb_cloud_key *ck, tfheb_params *out);

/* Files in the reference's format (tfhe_io.cpp): what one side writes, the other reads.
 *   tfheb_params_save / _load          export_tfheGateBootstrappingParameterSet_toFile /
 *                                      new_tfheGateBootstrappingParameterSet_fromFile (:1036-1049)
 *   tfheb_cloud_key_save / _load       export_ / new_tfheGateBootstrappingCloudKeySet_..File (:1125-1136)
 *   tfheb_secret_keyset_save / _load   export_ / new_tfheGateBootstrappingSecretKeySet_..File (:1179-1190)
 *   tfheb_ciphertexts_save / _load     export_gate_bootstrapping_ciphertext_toFile /
 *                                      import_gate_bootstrapping_ciphertext_fromFile (:1211-1220),
 *                                      `count` samples back to back, [count][n+1] int32; variances
 *                                      may be NULL (saved as 0, not returned).
 * A parameter file stores reals with 8 decimals ("%.8lf"), so a loaded ks_stdev / bk_stdev is the
 * rounded value, as in the reference.  Loading checks section titles and block type ids and
 * returns TFHEB_ERR_INVALID (with tfheb_last_error) where the reference aborts. */
tfheb_status tfheb_params_save(const char *path, const tfheb_params *p);
tfheb_status tfheb_params_load(const char *path, tfheb_params *p);
tfheb_status tfheb_cloud_key_save(const tfheb_cloud_key *ck, const char *path);
tfheb_status tfheb_cloud_key_load(const char *path, tfheb_cloud_key **ck);
tfheb_status tfheb_secret_keyset_save(const tfheb_secret_key *sk, const tfheb_cloud_key *ck, const char *path);
tfheb_status tfheb_secret_keyset_load(const char *path, tfheb_secret_key **sk, tfheb_cloud_key **ck);
tfheb_status tfheb_ciphertexts_save(const char *path, const tfheb_params *p, int32_t count, const int32_t *cts,
                                    const double *variances);
tfheb_status tfheb_ciphertexts_load(const char *path, const tfheb_params *p, int32_t count, int32_t *cts,
                                    double *variances);

/* Replaces delete_gate_bootstrapping_{secret,cloud}_keyset (tfhe_gate_bootstrapping.cpp:111-130). */
void tfheb_secret_key_free(tfheb_secret_key *sk);
void tfheb_cloud_key_free(tfheb_cloud_key *ck);

/* Replaces bootsSymEncrypt / bootsSymDecrypt (tfhe_gate_bootstrapping.cpp:154-165):
 * bits -> [count][n+1] with noise stdev ks_stdev; decrypt returns bits and optional raw phases. */
tfheb_status tfheb_encrypt(const tfheb_secret_key *sk, const int32_t *bits, int32_t count, uint64_t seed,
                           int32_t *out);
tfheb_status tfheb_decrypt(const tfheb_secret_key *sk, const int32_t *cts, int32_t count, int32_t *bits,
                           int32_t *phases);

/* Replaces lweSymEncrypt / lweSymDecrypt (lwe-functions.cpp:33-44, 86-90) for batches: torus
 * messages mu[count] -> [count][n+1] with noise stdev `stdev`; decryption returns each phase
 * rounded to the nearest multiple of 1/msize (approxPhase, numeric-functions.cpp:45-53). */
tfheb_status tfheb_encrypt_torus(const tfheb_secret_key *sk, const int32_t *mu, int32_t count, double stdev,
                                 uint64_t seed, int32_t *out);
tfheb_status tfheb_decrypt_torus(const tfheb_secret_key *sk, const int32_t *cts, int32_t count, int32_t msize,
                                 int32_t *out);

/* Moves the cloud key to a GPU: FFT-domain bootstrapping key in the requested precisions
 * (bit 0 = FP64, bit 1 = split FP32), keyswitching key, twiddle tables.  The FFT-domain key is
 * computed on the GPU with FP64 transforms, replacing init_LweBootstrappingKeyFFT
 * (lwe-bootstrapping-functions-fft.cpp:23-52).
 * split_shift: weight 2^split_shift of the high limb in split mode (0 = the parameter-dependent
 * default of tfheb_default_split_shift). */
tfheb_status tfheb_cloud_key_to_device(tfheb_cloud_key *ck, int32_t device, int32_t precision_mask,
                                       int32_t split_shift);

/* Copies the device FFT-domain bootstrapping key of `precision` to host memory (`bytes` must be
 * n*(k+1)*l*(k+1)*N/2*16).  Per key polynomial, spectrum / M in slot order (tfheb_fft_slot_order):
 *   FP64:  [8][N/16] double2 (re, im)
 *   split: [4][2][N/16] float4 {re(2m), re(2m+1), im(2m), im(2m+1)} for register pair m and limb
 *          (0 = hi, 1 = lo of c = hi * 2^S + lo).
 * For tests and tooling; no reference counterpart. */
tfheb_status tfheb_cloud_key_fft_download(const tfheb_cloud_key *ck, int32_t precision, void *out, size_t bytes);

/* Batched gates on host buffers ([count][n+1] each; c only for MUX, b unused for NOT/COPY):
 * the batched counterpart of bootsNAND...bootsMUX (boot-gates.cpp:34-370).  Synchronous. */
tfheb_status tfheb_gate_batch(tfheb_cloud_key *ck, int32_t gate, int32_t precision, int32_t count,
                              const int32_t *a, const int32_t *b, const int32_t *c, int32_t *out);

/* tfheb_gate_batch plus, per gate, the number of keyswitching-key rows its keyswitch subtracted
 * (the non-zero digits of lweKeySwitchTranslate_fromArray, lwe-keyswitch-functions.cpp:114-129):
 * the reference's result current_variance is the sum of that many key-sample variances.  NOT and
 * COPY report -1 (no keyswitch: the input's variance carries over, lwe-functions.cpp:111-126). */
tfheb_status tfheb_gate_batch_terms(tfheb_cloud_key *ck, int32_t gate, int32_t precision, int32_t count,
                                    const int32_t *a, const int32_t *b, const int32_t *c, int32_t *out,
                                    int32_t *terms);

/* The same batch sharded across several keys, each moved to its own GPU with
 * tfheb_cloud_key_to_device (keys with the same key material; the same device twice is allowed).
 * Shard k is rows [count*k/nkeys, count*(k+1)/nkeys), evaluated with tfheb_gate_batch on key k in
 * its own host thread; the output is bit-identical to one tfheb_gate_batch call.  Replica
 * sharding only: gates of a batch are independent, so there is no exchange between GPUs.
 * No reference counterpart (the reference evaluates gates on one CPU thread per call).  On error
 * the message names the failing shard. */
tfheb_status tfheb_gate_batch_multi(tfheb_cloud_key *const *cks, int32_t nkeys, int32_t gate, int32_t precision,
                                    int32_t count, const int32_t *a, const int32_t *b, const int32_t *c,
                                    int32_t *out);

/* Same on device buffers, enqueued on `stream` (a cudaStream_t, NULL = the key's stream).  Every
 * buffer must be device (or managed) memory on the key's GPU (TFHEB_ERR_INVALID otherwise); this holds
 * for all *_device calls below.  Calls on one key may use different streams: those that use the
 * key's scratch (this one, the bootstrap calls, tfheb_gate_batch) run on the GPU in call order, each
 * waiting on the device for the previous one, and a netlist's runs likewise. */
tfheb_status tfheb_gate_batch_device(tfheb_cloud_key *ck, int32_t gate, int32_t precision, int32_t count,
                                     const int32_t *d_a, const int32_t *d_b, const int32_t *d_c, int32_t *d_out,
                                     void *stream);

/* Mixed gate types in one batch on a device wire array (no reference counterpart; the reference
 * calls the gate functions of boot-gates.cpp one at a time).  d_wires holds num_wires rows of n+1
 * int32.  Gate g (code gates[g]) reads rows idx_a[g], idx_b[g] (binary gates and MUX) and idx_c[g]
 * (MUX) and writes row out_idx[g]; NOT/COPY read idx_a only.  Every operand is read before any
 * output is written, so an output may overwrite an operand of the same batch.  The index arrays are
 * host arrays, checked on the host (rows in range, no output row twice) and uploaded on each call;
 * scratch is stream-ordered (cudaMallocAsync / cudaFreeAsync).  Asynchronous on `stream` (NULL: the
 * key's stream). */
tfheb_status tfheb_gate_batch_mixed_device(tfheb_cloud_key *ck, int32_t precision, int32_t count,
                                           const int32_t *gates, const int32_t *idx_a, const int32_t *idx_b,
                                           const int32_t *idx_c, const int32_t *out_idx, int32_t *d_wires,
                                           int32_t num_wires, void *stream);

/* Hot-path pieces on device buffers (the scalar reference functions, batched):
 *   tfheb_bootstrap_woks_device  -> tfhe_bootstrap_woKS_FFT (lwe-bootstrapping-functions-fft.cpp:169-200)
 *                                    in [count][n+1] -> out [count][k*N+1]
 *   tfheb_bootstrap_device       -> tfhe_bootstrap_FFT (lwe-bootstrapping-functions-fft.cpp:213-225)
 *                                    in [count][n+1] -> out [count][n+1]
 *   tfheb_blind_rotate_device    -> tfhe_blindRotate_FFT (lwe-bootstrapping-functions-fft.cpp:88-112)
 *                                    acc [count][k+1][N] in place, bara [count][nsteps] (values in [0,2N))
 *   tfheb_keyswitch_device       -> lweKeySwitch (lwe-keyswitch-functions.cpp:228-238)
 *                                    in [count][k*N+1] -> out [count][n+1]                    */
tfheb_status tfheb_bootstrap_woks_device(tfheb_cloud_key *ck, int32_t precision, int32_t mu, int32_t count,
                                         const int32_t *d_in, int32_t *d_out, void *stream);
tfheb_status tfheb_bootstrap_device(tfheb_cloud_key *ck, int32_t precision, int32_t mu, int32_t count,
                                    const int32_t *d_in, int32_t *d_out, void *stream);
tfheb_status tfheb_blind_rotate_device(tfheb_cloud_key *ck, int32_t precision, int32_t count, int32_t nsteps,
                                       const int32_t *d_bara, int32_t *d_acc, void *stream);
tfheb_status tfheb_keyswitch_device(tfheb_cloud_key *ck, int32_t count, const int32_t *d_in, int32_t *d_out,
                                    void *stream);

/* The remaining scalar blind-rotation entry points, batched on device buffers:
 *   tfheb_blind_rotate_steps_device   -> tfhe_blindRotate_FFT (lwe-bootstrapping-functions-fft.cpp:88-112)
 *       over the key's TGSW samples first_step .. first_step+nsteps-1: acc [count][k+1][N] in place,
 *       bara [count][nsteps] (values taken mod 2N)
 *   tfheb_blind_rotate_extract_device -> tfhe_blindRotateAndExtract_FFT (:127-156): acc = (0,
 *       X^{2N-barb} v) from v [count][N] and barb [count], the same rotation, then the sample
 *       extraction at index 0 (lwe.cpp:41-53) into out [count][k*N+1]
 *   tfheb_extern_product_device       -> tGswExternProduct (tgsw-functions.cpp:416-431) with the key's
 *       TGSW sample `step`: out = bk_step (x) in, in/out [count][k+1][N] (may be the same buffer)
 *   tfheb_ks_terms_device             -> the digit count of lweKeySwitch (lwe-keyswitch-functions.cpp:
 *       114-129): terms [count] = non-zero digits of each extracted sample in [count][k*N+1]
 * Asynchronous on `stream` (NULL: the key's stream), like the device calls above. */
tfheb_status tfheb_blind_rotate_steps_device(tfheb_cloud_key *ck, int32_t precision, int32_t count, int32_t first_step,
                                             int32_t nsteps, const int32_t *d_bara, int32_t *d_acc, void *stream);
tfheb_status tfheb_blind_rotate_extract_device(tfheb_cloud_key *ck, int32_t precision, int32_t count,
                                               int32_t first_step, int32_t nsteps, const int32_t *d_v,
                                               const int32_t *d_barb, const int32_t *d_bara, int32_t *d_out,
                                               void *stream);
tfheb_status tfheb_extern_product_device(tfheb_cloud_key *ck, int32_t precision, int32_t count, int32_t step,
                                         const int32_t *d_in, int32_t *d_out, void *stream);
tfheb_status tfheb_ks_terms_device(tfheb_cloud_key *ck, int32_t count, const int32_t *d_in, int32_t *d_terms,
                                   void *stream);

/* Synchronise the key's stream and report any pending device error (TFHEB_ERR_TIMEOUT when a
 * bounded device-side wait of a kernel ran out). */
tfheb_status tfheb_synchronize(tfheb_cloud_key *ck);

/* Limit of every device-side wait of the key's kernels (default 1 s).  The reference has no
 * device waits; this is the failure-detection knob of the GPU engine. */
tfheb_status tfheb_set_wait_timeout(tfheb_cloud_key *ck, uint64_t timeout_ns);

/* Failure-detection test hook: when set, the blind rotation's key-streaming warp and the
 * keyswitch kernels' copy-issuing thread issue no copies, so every consumer wait runs out after the
 * timeout and the launch reports TFHEB_ERR_TIMEOUT (from the call or from tfheb_synchronize) with
 * the context still usable.  No reference counterpart. */
tfheb_status tfheb_test_stall_key_stream(tfheb_cloud_key *ck, int32_t stall);

/* Per-kernel timing: when enabled, every kernel the key launches is bracketed by CUDA events on
 * its stream.  read: ms[4] / launches[4] accumulated for prologue, blind rotation, extraction,
 * keyswitch (reset != 0 clears the totals).  No reference counterpart (the reference has no
 * instrumentation beyond clock() in its test programs). */
tfheb_status tfheb_profile(tfheb_cloud_key *ck, int32_t enable);
tfheb_status tfheb_profile_read(tfheb_cloud_key *ck, double *ms, int64_t *launches, int32_t reset);

/* FP32 (precision 1) or FP64 (precision 0) fused multiply-add throughput of the device in TFLOP/s,
 * measured by a dependent-chain probe kernel: the CUDA-core roofline denominator. */
tfheb_status tfheb_measure_fma_peak(int32_t device, int32_t precision, double *tflops);

/* Tensor cores or CUDA cores for a radix-8 stage of the FFT: applies 8-point complex DFTs to
 * register-resident data over the whole GPU and reports the device time per DFT and the largest
 * error relative to the column norm against FP64 DFTs.  method 0 = the FFT's dft8 codelet on the
 * CUDA cores; 1 = the DFT as a 16x16 real matrix product with mma.sync m16n8k8 TF32 in three
 * passes (FP32-level accuracy), operands kept in their fragment layouts (compute only); 2 = as 1,
 * plus the warp shuffles that move each result into the next stage's operand layout.  No reference
 * counterpart (the reference's FFT is AVX code on the CPU, spqlios-fft-fma.s). */
tfheb_status tfheb_measure_dft8(int32_t device, int32_t method, double *ns_per_dft, double *max_rel_err);

/* Blind-rotation launch variants an autotuner chooses from, for ring degree N, gadget length l = 3
 * (the 128-bit and N = 2048 sets) and a precision: bootstraps per CTA (teams_per_cta) and key-ring
 * depth; *count receives how many exist (arrays filled up to cap).  Two entries may share both
 * numbers: one streams the key with a dedicated warp, the other from its first thread.  tfheb_cloud_key_br_variants
 * lists them for a key's own parameter set (the 80-bit set has l = 2).  tfheb_set_br_variant picks
 * one for a key; tfheb_autotune times them all on `boots` synthetic bootstraps, keeps the fastest
 * for the key, and writes each variant's time to ms[] (up to cap).  It then times, for each g below
 * the winner's bootstraps per CTA, every compiled variant that fits a full wave of SMs x g bootstraps
 * and keeps the fastest for such one-wave batches (without autotuning, one-wave batches use the
 * variant with the fewest bootstraps per CTA that fits; at one per CTA, the variant that spreads a
 * bootstrap's gadget digits over one team each, N = 1024).  Results never depend on the variant.  No
 * reference counterpart (the reference has one CPU code path). */
tfheb_status tfheb_br_variants(int32_t N, int32_t precision, int32_t *teams_per_cta, int32_t *ring_depth,
                               int32_t cap, int32_t *count);
tfheb_status tfheb_cloud_key_br_variants(const tfheb_cloud_key *ck, int32_t precision, int32_t *teams_per_cta,
                                         int32_t *ring_depth, int32_t cap, int32_t *count);
/* FFT plan of each variant of tfheb_cloud_key_br_variants, same order: 0 = the radix-8 team FFT with
 * one transform per thread; 1 = the same transform, two per thread on packed f32x2, with the digit
 * spectra parked in tensor memory and the multiply-accumulate one output polynomial at a time
 * (split-FP32; the same bits as plan 0).  The autotuner times both plans. */
tfheb_status tfheb_cloud_key_br_plans(const tfheb_cloud_key *ck, int32_t precision, int32_t *plan, int32_t cap,
                                      int32_t *count);
tfheb_status tfheb_set_br_variant(tfheb_cloud_key *ck, int32_t precision, int32_t variant);
tfheb_status tfheb_autotune(tfheb_cloud_key *ck, int32_t precision, int32_t boots, double *ms, int32_t cap);

/* Keyswitch kernel of a key: 0 = default, 1 = one CTA per sample, 2 = tiled (key rows shared
 * through shared memory), 3 = register-key (key rows held in registers across samples),
 * 4 = tensor-core (the digit selection as an int8 one-hot product with the key's byte planes on
 * tcgen05.mma); 2 to 4 need ks_t = 8 and basebit = 2 (TFHEB_ERR_UNSUPPORTED otherwise), which the
 * default also uses when it can.  All give the reference's lweKeySwitch result bit for bit; the
 * choice is a performance knob.  No reference counterpart. */
tfheb_status tfheb_set_keyswitch_kernel(tfheb_cloud_key *ck, int32_t which);

/* Weight exponent S of the high limb the split-FP32 key uses by default for a parameter set. */
int32_t tfheb_default_split_shift(const tfheb_params *p);

/* Levelled netlist evaluation.  No counterpart in the reference, whose callers chain single gate
 * calls (test-long-run.cpp:61-185, test-addition-boot.cpp).  Wires 0..num_inputs-1 are primary
 * inputs; gate g (codes as above, topological order) produces wire num_inputs+g and reads wires
 * in_a[g], in_b[g] (and in_c[g] for MUX; only in_a for NOT/COPY), each below num_inputs+g.
 * create: levels the gates (as many levels as the critical path; gates with slack move to levels
 * where they complete blind-rotation waves, one schedule per precision for the key's current
 * launch variants), uploads per-level descriptors and allocates the scratch of the widest level;
 * info reports the level count and the widest level of the split-FP32 schedule.  run: d_wires is a device array [num_inputs+num_gates][n+1] whose input rows the caller
 * filled; on return (stream-ordered) row num_inputs+g holds gate g's output.  With use_graph, the
 * first run on a (precision, d_wires) pair evaluates eagerly and captures the level sequence into a
 * CUDA graph; later runs replay that graph with one launch. */
typedef struct tfheb_netlist tfheb_netlist;
tfheb_status tfheb_netlist_create(tfheb_cloud_key *ck, int32_t num_inputs, int32_t num_gates, const int32_t *gates,
                                  const int32_t *in_a, const int32_t *in_b, const int32_t *in_c,
                                  tfheb_netlist **out);
tfheb_status tfheb_netlist_info(const tfheb_netlist *nl, int32_t *num_levels, int32_t *max_width);
tfheb_status tfheb_netlist_run(tfheb_netlist *nl, int32_t precision, int32_t *d_wires, int32_t use_graph,
                               void *stream);
void tfheb_netlist_free(tfheb_netlist *nl);

/* The same netlist sharded across several cloud keys, each on its own GPU (replica sharding of
 * netlist levels; no reference counterpart).  The keys must be distinct, share one parameter set
 * and be on their devices (two keys may share a device).  create: one level assignment for all keys,
 * packed for their waves together; every level's bootstrapped gates are cut into one contiguous run
 * per key with balanced bootstrap counts (a MUX counts two); NOT/COPY gates run on every key.  Each key
 * holds a full wire array.  run: wires is a HOST array [num_inputs+num_gates][n+1] whose input rows the
 * caller filled; they are copied to every key.  Per level, every key evaluates its run on its own
 * stream, then copies those output rows into every other key's wire array (peer copies; the next
 * level waits on them with events, no host synchronisation between levels).  Returns when gate g's
 * output is in row num_inputs+g of `wires`, bit-identical to tfheb_netlist_run on one key.  Launches
 * are eager (no CUDA graph). */
typedef struct tfheb_netlist_multi tfheb_netlist_multi;
tfheb_status tfheb_netlist_multi_create(tfheb_cloud_key *const *cks, int32_t nkeys, int32_t num_inputs,
                                        int32_t num_gates, const int32_t *gates, const int32_t *in_a,
                                        const int32_t *in_b, const int32_t *in_c, tfheb_netlist_multi **out);
tfheb_status tfheb_netlist_multi_run(tfheb_netlist_multi *nl, int32_t precision, int32_t *wires);
void tfheb_netlist_multi_free(tfheb_netlist_multi *nl);

/* Allocation-free variant of tfheb_gate_batch_device, for callers that cannot call cudaMalloc
 * (real-time or signal-handling code that must not enter the allocator, or a process whose device
 * memory belongs to a framework's pool).  No counterpart in the reference, which has no device
 * memory at all.  All scratch comes from one fixed 8 MiB device array in the library, so a call
 * allocates and frees nothing; it fits 565 binary / 327 MUX gates at the default parameters (301 /
 * 176 at N=2048) and rejects larger counts with TFHEB_ERR_INVALID.  Buffers are checked like
 * tfheb_gate_batch_device's.  The array is shared by all calls on a device: calls that overlap on
 * the GPU race, so keep them on one stream.  The first call on a device looks up the array's
 * address; make it before any stream capture.  That address belongs to the device's context, so do
 * not call this again on a device after cudaDeviceReset.  The key must already be on the device
 * (tfheb_cloud_key_to_device). */
tfheb_status tfheb_gate_batch_device_noalloc(tfheb_cloud_key *ck, int32_t gate, int32_t precision, int32_t count,
                                             const int32_t *d_a, const int32_t *d_b, const int32_t *d_c,
                                             int32_t *d_out, void *stream);

/* Layout helpers (host only, no GPU): slot order of the FFT-domain key for ring degree N
 * (slot_freq[R*N/16]: frequency held by register r of thread t at index r*(N/16)+t). */
tfheb_status tfheb_fft_slot_order(int32_t N, int32_t *slot_freq);

#ifdef __cplusplus
}
#endif
#endif
