// Test-infrastructure shim over the reference library (tfhe v1.1, spqlios-fma backend) built
// from its own sources by oracle/ref.mk into oracle/_ref/.  Everything here is a thin extern "C"
// wrapper, so that pytest (ctypes) can drive the reference on raw int32 buffers:
//   * seeded key generation and raw key export (to import identical keys into the GPU engine),
//   * the reference gates, bootstrap and keyswitch on identical inputs (parity checker),
//   * small building blocks (decomposition, rotation, extraction, mod-switch) for golden vectors,
//   * the multi-threaded CPU baseline (one gate per thread; FFT processors are thread_local in
//     the reference, fft_processor_spqlios.cpp:123).
// Nothing in the product library links or loads this file.
#include <tfhe.h>
#include <tfhe_io.h>
#include <tfhe_gate_bootstrapping_structures.h>
#include <lwekey.h>
#include <lweparams.h>
#include <lwesamples.h>
#include <lwekeyswitch.h>
#include <lwebootstrappingkey.h>
#include <tlwe.h>
#include <tgsw.h>
#include <polynomials.h>
#include <tgsw_functions.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cstring>
#include <thread>
#include <vector>

namespace {

struct RsKeys {
    TFheGateBootstrappingParameterSet *params;
    TFheGateBootstrappingSecretKeySet *sk;
};

inline const LweParams *io_params(const RsKeys *k) { return k->params->in_out_params; }
inline const TGswParams *bk_params(const RsKeys *k) { return k->params->tgsw_params; }
inline const TLweParams *acc_params(const RsKeys *k) { return k->params->tgsw_params->tlwe_params; }

void load_lwe(LweSample *s, const int32_t *raw, int32_t n) {
    std::memcpy(s->a, raw, sizeof(int32_t) * n);
    s->b = raw[n];
    s->current_variance = 0.;
}

void store_lwe(int32_t *raw, const LweSample *s, int32_t n) {
    std::memcpy(raw, s->a, sizeof(int32_t) * n);
    raw[n] = s->b;
}

void run_gate(int gate, LweSample *r, const LweSample *a, const LweSample *b, const LweSample *c,
              const TFheGateBootstrappingCloudKeySet *ck) {
    switch (gate) {
        case 0: bootsNAND(r, a, b, ck); break;
        case 1: bootsOR(r, a, b, ck); break;
        case 2: bootsAND(r, a, b, ck); break;
        case 3: bootsXOR(r, a, b, ck); break;
        case 4: bootsXNOR(r, a, b, ck); break;
        case 5: bootsNOR(r, a, b, ck); break;
        case 6: bootsANDNY(r, a, b, ck); break;
        case 7: bootsANDYN(r, a, b, ck); break;
        case 8: bootsORNY(r, a, b, ck); break;
        case 9: bootsORYN(r, a, b, ck); break;
        case 10: bootsMUX(r, a, b, c, ck); break;
        case 11: bootsNOT(r, a, ck); break;
        case 12: bootsCOPY(r, a, ck); break;
        default: break;
    }
}

}  // namespace

extern "C" {

void rs_seed(uint32_t seed) {
    uint32_t v[1] = {seed};
    tfhe_random_generator_setSeed(v, 1);
}

// custom == 0: the reference's default 128-bit parameter set (tfhe_gate_bootstrapping.cpp:51-75).
void *rs_keygen(int custom, int n, int N, int k, int l, int Bgbit, int ks_t, int ks_basebit,
                double ks_stdev, double bk_stdev, uint32_t seed) {
    rs_seed(seed);
    RsKeys *keys = new RsKeys();
    if (!custom) {
        keys->params = new_default_gate_bootstrapping_parameters(110);
    } else {
        LweParams *in = new_LweParams(n, ks_stdev, 0.012467);
        TLweParams *acc = new_TLweParams(N, k, bk_stdev, 0.012467);
        TGswParams *bk = new_TGswParams(l, Bgbit, acc);
        keys->params = new TFheGateBootstrappingParameterSet(ks_t, ks_basebit, in, bk);
    }
    keys->sk = new_random_gate_bootstrapping_secret_keyset(keys->params);
    return keys;
}

void rs_free(void *h) {
    RsKeys *keys = static_cast<RsKeys *>(h);
    delete_gate_bootstrapping_secret_keyset(keys->sk);
    delete keys;
}

// out: n, N, k, l, Bgbit, ks_t, ks_basebit, kpl
void rs_dims(void *h, int32_t *out) {
    RsKeys *keys = static_cast<RsKeys *>(h);
    out[0] = io_params(keys)->n;
    out[1] = acc_params(keys)->N;
    out[2] = acc_params(keys)->k;
    out[3] = bk_params(keys)->l;
    out[4] = bk_params(keys)->Bgbit;
    out[5] = keys->params->ks_t;
    out[6] = keys->params->ks_basebit;
    out[7] = bk_params(keys)->kpl;
}

// Raw key export.
//   lwe_key  [n]
//   tlwe_key [k][N]
//   ksk      [k*N][t][base][n+1]     (a[0..n-1], b)   -- LweKeySwitchKey::ks0_raw order
//   bsk      [n][kpl][k+1][N]        coefficient-domain TGSW rows (TGswSample::all_sample)
void rs_export(void *h, int32_t *lwe_key, int32_t *tlwe_key, int32_t *ksk, int32_t *bsk) {
    RsKeys *keys = static_cast<RsKeys *>(h);
    const int32_t n = io_params(keys)->n;
    const int32_t N = acc_params(keys)->N;
    const int32_t k = acc_params(keys)->k;
    const int32_t kpl = bk_params(keys)->kpl;
    if (lwe_key) std::memcpy(lwe_key, keys->sk->lwe_key->key, sizeof(int32_t) * n);
    if (tlwe_key)
        for (int32_t i = 0; i < k; i++)
            std::memcpy(tlwe_key + i * N, keys->sk->tgsw_key->tlwe_key.key[i].coefs, sizeof(int32_t) * N);
    const LweBootstrappingKey *bk = keys->sk->cloud.bk;
    if (ksk) {
        const LweKeySwitchKey *ks = bk->ks;
        const int64_t rows = int64_t(ks->n) * ks->t * ks->base;
        for (int64_t r = 0; r < rows; r++) store_lwe(ksk + r * (n + 1), ks->ks0_raw + r, n);
    }
    if (bsk) {
        int64_t off = 0;
        for (int32_t i = 0; i < n; i++)
            for (int32_t p = 0; p < kpl; p++)
                for (int32_t u = 0; u <= k; u++) {
                    std::memcpy(bsk + off, bk->bk[i].all_sample[p].a[u].coefsT, sizeof(int32_t) * N);
                    off += N;
                }
    }
}

void rs_encrypt(void *h, int32_t count, const int32_t *bits, int32_t *out) {
    RsKeys *keys = static_cast<RsKeys *>(h);
    const int32_t n = io_params(keys)->n;
    LweSample *s = new_gate_bootstrapping_ciphertext(keys->params);
    for (int32_t g = 0; g < count; g++) {
        bootsSymEncrypt(s, bits[g], keys->sk);
        store_lwe(out + int64_t(g) * (n + 1), s, n);
    }
    delete_gate_bootstrapping_ciphertext(s);
}

void rs_decrypt(void *h, int32_t count, const int32_t *in, int32_t *bits, int32_t *phases) {
    RsKeys *keys = static_cast<RsKeys *>(h);
    const int32_t n = io_params(keys)->n;
    LweSample *s = new_gate_bootstrapping_ciphertext(keys->params);
    for (int32_t g = 0; g < count; g++) {
        load_lwe(s, in + int64_t(g) * (n + 1), n);
        if (bits) bits[g] = bootsSymDecrypt(s, keys->sk);
        if (phases) phases[g] = lwePhase(s, keys->sk->lwe_key);
    }
    delete_gate_bootstrapping_ciphertext(s);
}

// gate codes: 0 NAND 1 OR 2 AND 3 XOR 4 XNOR 5 NOR 6 ANDNY 7 ANDYN 8 ORNY 9 ORYN 10 MUX 11 NOT 12 COPY
void rs_gate(void *h, int gate, int32_t count, const int32_t *a, const int32_t *b, const int32_t *c,
             int32_t *out) {
    RsKeys *keys = static_cast<RsKeys *>(h);
    const int32_t n = io_params(keys)->n;
    LweSample *sa = new_gate_bootstrapping_ciphertext(keys->params);
    LweSample *sb = new_gate_bootstrapping_ciphertext(keys->params);
    LweSample *sc = new_gate_bootstrapping_ciphertext(keys->params);
    LweSample *sr = new_gate_bootstrapping_ciphertext(keys->params);
    for (int32_t g = 0; g < count; g++) {
        const int64_t off = int64_t(g) * (n + 1);
        load_lwe(sa, a + off, n);
        if (b) load_lwe(sb, b + off, n);
        if (c) load_lwe(sc, c + off, n);
        run_gate(gate, sr, sa, sb, sc, &keys->sk->cloud);
        store_lwe(out + off, sr, n);
    }
    delete_gate_bootstrapping_ciphertext(sr);
    delete_gate_bootstrapping_ciphertext(sc);
    delete_gate_bootstrapping_ciphertext(sb);
    delete_gate_bootstrapping_ciphertext(sa);
}

// tfhe_bootstrap_woKS_FFT on raw inputs [count][n+1] -> outputs [count][k*N+1]
void rs_bootstrap_woks(void *h, int32_t mu, int32_t count, const int32_t *in, int32_t *out) {
    RsKeys *keys = static_cast<RsKeys *>(h);
    const int32_t n = io_params(keys)->n;
    const LweParams *ext = &acc_params(keys)->extracted_lweparams;
    const int32_t kN = ext->n;
    LweSample *x = new_LweSample(io_params(keys));
    LweSample *u = new_LweSample(ext);
    for (int32_t g = 0; g < count; g++) {
        load_lwe(x, in + int64_t(g) * (n + 1), n);
        tfhe_bootstrap_woKS_FFT(u, keys->sk->cloud.bkFFT, mu, x);
        store_lwe(out + int64_t(g) * (kN + 1), u, kN);
    }
    delete_LweSample(u);
    delete_LweSample(x);
}

// lweKeySwitch on raw inputs [count][k*N+1] -> [count][n+1], with each result's current_variance
// (the keyswitching key's sample variances summed over the non-zero digits,
// lwe-keyswitch-functions.cpp:114-129) into var[count] when var is not null.  The samples are spread
// over the host's threads; lweKeySwitch keeps no shared state.
void rs_keyswitch(void *h, int32_t count, const int32_t *in, int32_t *out, double *var) {
    RsKeys *keys = static_cast<RsKeys *>(h);
    const int32_t n = io_params(keys)->n;
    const LweParams *ext = &acc_params(keys)->extracted_lweparams;
    const int32_t kN = ext->n;
    const int32_t threads = std::max(1, std::min<int32_t>(count, (int32_t)std::thread::hardware_concurrency()));
    auto work = [&](int32_t t) {
        LweSample *x = new_LweSample(ext);
        LweSample *r = new_LweSample(io_params(keys));
        for (int32_t g = t; g < count; g += threads) {
            load_lwe(x, in + int64_t(g) * (kN + 1), kN);
            lweKeySwitch(r, keys->sk->cloud.bkFFT->ks, x);
            store_lwe(out + int64_t(g) * (n + 1), r, n);
            if (var) var[g] = r->current_variance;
        }
        delete_LweSample(r);
        delete_LweSample(x);
    };
    std::vector<std::thread> pool;
    for (int32_t t = 1; t < threads; t++) pool.emplace_back(work, t);
    work(0);
    for (auto &th : pool) th.join();
}

// ---- building blocks (no keys needed) ---------------------------------------------------------

int32_t rs_modswitch_from(int32_t phase, int32_t Msize) { return modSwitchFromTorus32(phase, Msize); }
int32_t rs_modswitch_to(int32_t mu, int32_t Msize) { return modSwitchToTorus32(mu, Msize); }
int32_t rs_dtot32(double d) { return dtot32(d); }

// tGswTorus32PolynomialDecompH: poly[N] -> digits[l][N]
void rs_decompose(int32_t N, int32_t l, int32_t Bgbit, const int32_t *poly, int32_t *digits) {
    TLweParams *tp = new_TLweParams(N, 1, 1e-9, 1e-2);
    TGswParams *gp = new_TGswParams(l, Bgbit, tp);
    TorusPolynomial *src = new_TorusPolynomial(N);
    IntPolynomial *dec = new_IntPolynomial_array(l, N);
    std::memcpy(src->coefsT, poly, sizeof(int32_t) * N);
    tGswTorus32PolynomialDecompH(dec, src, gp);
    for (int32_t p = 0; p < l; p++) std::memcpy(digits + p * N, dec[p].coefs, sizeof(int32_t) * N);
    delete_IntPolynomial_array(l, dec);
    delete_TorusPolynomial(src);
    delete_TGswParams(gp);
    delete_TLweParams(tp);
}

// torusPolynomialMulByXaiMinusOne (rot=0) / torusPolynomialMulByXai (rot=1)
void rs_rotate(int32_t N, int32_t a, int32_t minus_one, const int32_t *in, int32_t *out) {
    TorusPolynomial *src = new_TorusPolynomial(N);
    TorusPolynomial *dst = new_TorusPolynomial(N);
    std::memcpy(src->coefsT, in, sizeof(int32_t) * N);
    if (minus_one) torusPolynomialMulByXaiMinusOne(dst, a, src);
    else torusPolynomialMulByXai(dst, a, src);
    std::memcpy(out, dst->coefsT, sizeof(int32_t) * N);
    delete_TorusPolynomial(dst);
    delete_TorusPolynomial(src);
}

// tLweExtractLweSampleIndex(index 0): tlwe[(k+1)][N] -> lwe[k*N+1]
void rs_extract(int32_t N, int32_t k, const int32_t *tlwe, int32_t *out) {
    TLweParams *tp = new_TLweParams(N, k, 1e-9, 1e-2);
    TLweSample *x = new_TLweSample(tp);
    LweSample *r = new_LweSample(&tp->extracted_lweparams);
    for (int32_t u = 0; u <= k; u++) std::memcpy(x->a[u].coefsT, tlwe + u * N, sizeof(int32_t) * N);
    tLweExtractLweSample(r, x, &tp->extracted_lweparams, tp);
    store_lwe(out, r, k * N);
    delete_LweSample(r);
    delete_TLweSample(x);
    delete_TLweParams(tp);
}

// Polynomial products: 0 = FFT (spqlios, N=1024 only), 1 = Karatsuba, 2 = naive.
void rs_poly_mult(int32_t kind, int32_t N, const int32_t *ipoly, const int32_t *tpoly, int32_t *out) {
    IntPolynomial *a = new_IntPolynomial(N);
    TorusPolynomial *b = new_TorusPolynomial(N);
    TorusPolynomial *r = new_TorusPolynomial(N);
    std::memcpy(a->coefs, ipoly, sizeof(int32_t) * N);
    std::memcpy(b->coefsT, tpoly, sizeof(int32_t) * N);
    if (kind == 0) torusPolynomialMultFFT(r, a, b);
    else if (kind == 1) torusPolynomialMultKaratsuba(r, a, b);
    else torusPolynomialMultNaive(r, a, b);
    std::memcpy(out, r->coefsT, sizeof(int32_t) * N);
    delete_TorusPolynomial(r);
    delete_TorusPolynomial(b);
    delete_IntPolynomial(a);
}

// ---- CPU baseline ------------------------------------------------------------------------------
// Runs `gates_per_thread` gates of type `gate` on each of `threads` host threads, one gate per
// thread at a time, over inputs [threads*gates_per_thread][n+1] (c may be null for binary gates).
// Outputs go to out (same shape).  Returns wall-clock seconds of the evaluation only.
double rs_bench_gates(void *h, int gate, int32_t threads, int32_t gates_per_thread, const int32_t *a,
                      const int32_t *b, const int32_t *c, int32_t *out) {
    RsKeys *keys = static_cast<RsKeys *>(h);
    const int32_t n = io_params(keys)->n;
    std::atomic<int> ready{0};
    std::atomic<bool> go{false};
    std::vector<std::thread> pool;
    auto worker = [&](int32_t tid) {
        LweSample *sa = new_gate_bootstrapping_ciphertext(keys->params);
        LweSample *sb = new_gate_bootstrapping_ciphertext(keys->params);
        LweSample *sc = new_gate_bootstrapping_ciphertext(keys->params);
        LweSample *sr = new_gate_bootstrapping_ciphertext(keys->params);
        ready++;
        while (!go.load()) std::this_thread::yield();
        for (int32_t g = 0; g < gates_per_thread; g++) {
            const int64_t off = (int64_t(tid) * gates_per_thread + g) * (n + 1);
            load_lwe(sa, a + off, n);
            if (b) load_lwe(sb, b + off, n);
            if (c) load_lwe(sc, c + off, n);
            run_gate(gate, sr, sa, sb, sc, &keys->sk->cloud);
            store_lwe(out + off, sr, n);
        }
        delete_gate_bootstrapping_ciphertext(sr);
        delete_gate_bootstrapping_ciphertext(sc);
        delete_gate_bootstrapping_ciphertext(sb);
        delete_gate_bootstrapping_ciphertext(sa);
    };
    for (int32_t t = 0; t < threads; t++) pool.emplace_back(worker, t);
    while (ready.load() < threads) std::this_thread::yield();
    auto t0 = std::chrono::steady_clock::now();
    go.store(true);
    for (auto &th : pool) th.join();
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

}  // extern "C"

extern "C" {
// tGswExternProduct with the coefficient-domain bootstrapping-key sample i: out = bk_i (x) b, both
// [(k+1)][N], with b's current_variance b_var; the result's current_variance into *var
void rs_extern_product(void *h, int32_t i, const int32_t *b, double b_var, int32_t *out, double *var) {
    RsKeys *keys = static_cast<RsKeys *>(h);
    const TLweParams *tp = acc_params(keys);
    const int32_t N = tp->N, k = tp->k;
    TLweSample *x = new_TLweSample(tp);
    TLweSample *r = new_TLweSample(tp);
    for (int32_t u = 0; u <= k; u++) std::memcpy(x->a[u].coefsT, b + u * N, sizeof(int32_t) * N);
    x->current_variance = b_var;
    tGswExternProduct(r, keys->sk->cloud.bk->bk + i, x, bk_params(keys));
    for (int32_t u = 0; u <= k; u++) std::memcpy(out + u * N, r->a[u].coefsT, sizeof(int32_t) * N);
    *var = r->current_variance;
    delete_TLweSample(r);
    delete_TLweSample(x);
}

// tGswFFTExternMulToTLwe with bootstrapping-key row i: acc[(k+1)][N] <- bkFFT[i] (*) acc
void rs_extern_mul(void *h, int32_t i, int32_t *acc) {
    RsKeys *keys = static_cast<RsKeys *>(h);
    const TLweParams *tp = acc_params(keys);
    const int32_t N = tp->N, k = tp->k;
    TLweSample *x = new_TLweSample(tp);
    for (int32_t u = 0; u <= k; u++) std::memcpy(x->a[u].coefsT, acc + u * N, sizeof(int32_t) * N);
    tGswFFTExternMulToTLwe(x, keys->sk->cloud.bkFFT->bkFFT + i, bk_params(keys));
    for (int32_t u = 0; u <= k; u++) std::memcpy(acc + u * N, x->a[u].coefsT, sizeof(int32_t) * N);
    delete_TLweSample(x);
}
}

// ---- the reference's own file format (tfhe_io.cpp), through its FILE* functions -------------
extern "C" {

int rs_save_params(void *h, const char *path) {
    FILE *F = std::fopen(path, "wb");
    if (!F) return -1;
    export_tfheGateBootstrappingParameterSet_toFile(F, static_cast<RsKeys *>(h)->params);
    return std::fclose(F);
}

int rs_save_secret_keyset(void *h, const char *path) {
    FILE *F = std::fopen(path, "wb");
    if (!F) return -1;
    export_tfheGateBootstrappingSecretKeySet_toFile(F, static_cast<RsKeys *>(h)->sk);
    return std::fclose(F);
}

int rs_save_cloud_keyset(void *h, const char *path) {
    FILE *F = std::fopen(path, "wb");
    if (!F) return -1;
    export_tfheGateBootstrappingCloudKeySet_toFile(F, &static_cast<RsKeys *>(h)->sk->cloud);
    return std::fclose(F);
}

// count ciphertexts [count][n+1] with the given variances, back to back
int rs_save_ciphertexts(void *h, const char *path, int32_t count, const int32_t *raw, const double *variances) {
    RsKeys *keys = static_cast<RsKeys *>(h);
    const int32_t n = io_params(keys)->n;
    FILE *F = std::fopen(path, "wb");
    if (!F) return -1;
    LweSample *s = new_gate_bootstrapping_ciphertext(keys->params);
    for (int32_t g = 0; g < count; g++) {
        load_lwe(s, raw + (size_t)g * (n + 1), n);
        s->current_variance = variances[g];
        export_gate_bootstrapping_ciphertext_toFile(F, s, keys->params);
    }
    delete_gate_bootstrapping_ciphertext(s);
    return std::fclose(F);
}

int rs_load_ciphertexts(void *h, const char *path, int32_t count, int32_t *raw, double *variances) {
    RsKeys *keys = static_cast<RsKeys *>(h);
    const int32_t n = io_params(keys)->n;
    FILE *F = std::fopen(path, "rb");
    if (!F) return -1;
    LweSample *s = new_gate_bootstrapping_ciphertext(keys->params);
    for (int32_t g = 0; g < count; g++) {
        import_gate_bootstrapping_ciphertext_fromFile(F, s, keys->params);
        store_lwe(raw + (size_t)g * (n + 1), s, n);
        variances[g] = s->current_variance;
    }
    delete_gate_bootstrapping_ciphertext(s);
    return std::fclose(F);
}

// A key handle from a secret keyset file (parameters from the file, owned by the reference).
void *rs_load_secret_keyset(const char *path) {
    FILE *F = std::fopen(path, "rb");
    if (!F) return nullptr;
    RsKeys *keys = new RsKeys();
    keys->sk = new_tfheGateBootstrappingSecretKeySet_fromFile(F);
    keys->params = const_cast<TFheGateBootstrappingParameterSet *>(keys->sk->params);
    std::fclose(F);
    return keys;
}

}  // extern "C"
