/* A client of the reference's blind-rotation, external-product and keyswitch functions (tfhe.h:36-45,
 * tgsw_functions.h:40-46, lwe-functions.h:79), compiled as plain C against include/tfhe.h and linked
 * with libtfhe_b200.so.
 *
 *   dropin_rotate <secret keyset file> <record file> <precision 0|1>
 *
 * It loads a keyset written in the reference's file format and checks, bit for bit, that the entry
 * points agree with one another on the GPU:
 *   - tfhe_blindRotateAndExtract_FFT with the test vector [mu..mu] equals tfhe_bootstrap_woKS_FFT;
 *   - tfhe_blindRotate_FFT followed by the extraction formula (lwe.cpp:41-53) equals it as well;
 *   - tfhe_blindRotate on the keyset's coefficient-domain samples equals tfhe_blindRotate_FFT, and so
 *     does tfhe_blindRotate on a caller-made copy of those samples;
 *   - rotating over 5 samples at once equals rotating over 2 then 3;
 *   - acc + tGswExternProduct(bk_i, (X^a - 1) acc) equals one step of tfhe_blindRotate_FFT;
 *   - tGswExternMulToTLwe equals tGswExternProduct, with b's variance left out;
 *   - tfhe_bootstrap equals tfhe_bootstrap_FFT; lweKeySwitch of the extracted sample equals it too;
 *   - the extractions and rotations leave current_variance as the reference does.
 * It writes its inputs and outputs to the record file so that the caller can compare the keyswitch,
 * bootstrap, gate and external-product results, and their variances, with the reference library.
 * Exit status 0 when every check holds; a failing check prints its name. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "tfhe.h"

static int fails = 0;
static void check(const char *name, int ok) {
    if (!ok) {
        fprintf(stderr, "check failed: %s\n", name);
        fails++;
    }
}

static void put_i32(FILE *f, const int32_t *v, size_t n) { fwrite(v, sizeof(int32_t), n, f); }
static void put_lwe(FILE *f, const LweSample *s, int32_t n) {
    put_i32(f, s->a, (size_t)n);
    put_i32(f, &s->b, 1);
}
static void put_f64(FILE *f, double v) { fwrite(&v, sizeof(double), 1, f); }
static void put_tlwe(FILE *f, const TLweSample *s, int32_t k, int32_t N) {
    for (int32_t u = 0; u <= k; u++) put_i32(f, s->a[u].coefsT, (size_t)N);
}

static int same_lwe(const LweSample *x, const LweSample *y, int32_t n) {
    return memcmp(x->a, y->a, sizeof(int32_t) * (size_t)n) == 0 && x->b == y->b;
}
static int same_tlwe(const TLweSample *x, const TLweSample *y, int32_t k, int32_t N) {
    for (int32_t u = 0; u <= k; u++)
        if (memcmp(x->a[u].coefsT, y->a[u].coefsT, sizeof(int32_t) * (size_t)N) != 0) return 0;
    return 1;
}
static void copy_tlwe(TLweSample *dst, const TLweSample *src, int32_t k, int32_t N) {
    for (int32_t u = 0; u <= k; u++) memcpy(dst->a[u].coefsT, src->a[u].coefsT, sizeof(int32_t) * (size_t)N);
    dst->current_variance = src->current_variance;
}

static uint64_t rng = 0x9E3779B97F4A7C15ull;
static uint32_t next32(void) {
    rng ^= rng << 13;
    rng ^= rng >> 7;
    rng ^= rng << 17;
    return (uint32_t)(rng >> 16);
}

int main(int argc, char **argv) {
    if (argc < 4) {
        fprintf(stderr, "usage: dropin_rotate <secret keyset file> <record file> <precision 0|1>\n");
        return 2;
    }
    FILE *kf = fopen(argv[1], "rb");
    if (!kf) return 2;
    TFheGateBootstrappingSecretKeySet *key = new_tfheGateBootstrappingSecretKeySet_fromFile(kf);
    fclose(kf);
    FILE *rec = fopen(argv[2], "wb");
    if (!rec) return 2;
    tfhe_b200_set_precision(atoi(argv[3]));

    const TFheGateBootstrappingParameterSet *params = key->params;
    const TFheGateBootstrappingCloudKeySet *ck = &key->cloud;
    const TGswParams *gp = params->tgsw_params;
    const TLweParams *tp = gp->tlwe_params;
    const LweParams *io = params->in_out_params, *ext = &tp->extracted_lweparams;
    const int32_t n = io->n, N = tp->N, k = tp->k, kN = k * N, l = gp->l, kpl = gp->kpl;
    const Torus32 mu = modSwitchToTorus32(1, 8);

    LweSample *x = new_LweSample_array(2, io), *y = new_LweSample_array(4, io), *comb = new_LweSample(io);
    LweSample *u = new_LweSample_array(4, ext);
    TLweSample *acc = new_TLweSample_array(4, tp);
    TorusPolynomial *v = new_TorusPolynomial(N);
    int32_t *bara = (int32_t *)malloc(sizeof(int32_t) * (size_t)n);
    for (int32_t j = 0; j < N; j++) v->coefsT[j] = mu;

    const int trials = 3;
    for (int t = 0; t < trials; t++) {
        const int32_t bit0 = (int32_t)(next32() & 1), bit1 = (int32_t)(next32() & 1);
        bootsSymEncrypt(&x[0], bit0, key);
        bootsSymEncrypt(&x[1], bit1, key);
        put_lwe(rec, &x[0], n);
        put_lwe(rec, &x[1], n);

        /* bootstrap without keyswitch: the extraction leaves the variance as it was */
        u[0].current_variance = 12.5;
        tfhe_bootstrap_woKS_FFT(&u[0], ck->bkFFT, mu, &x[0]);
        check("woKS keeps the result's variance", u[0].current_variance == 12.5);
        put_lwe(rec, &u[0], kN);
        /* the same through blindRotateAndExtract_FFT from the mod-switched input */
        const int32_t barb = modSwitchFromTorus32(x[0].b, 2 * N);
        for (int32_t i = 0; i < n; i++) bara[i] = modSwitchFromTorus32(x[0].a[i], 2 * N);
        tfhe_blindRotateAndExtract_FFT(&u[1], v, ck->bkFFT->bkFFT, barb, bara, n, gp);
        check("blindRotateAndExtract_FFT == bootstrap_woKS_FFT", same_lwe(&u[1], &u[0], kN));
        /* ... and through blindRotate_FFT from (0, X^{2N-barb} v), then the extraction formula */
        const int32_t e = (2 * N - barb) % (2 * N);
        for (int32_t c = 0; c < k; c++) memset(acc[0].a[c].coefsT, 0, sizeof(int32_t) * (size_t)N);
        for (int32_t j = 0; j < N; j++) {
            int32_t src = j - e, neg = 0;
            while (src < 0) {
                src += N;
                neg ^= 1;
            }
            acc[0].b->coefsT[j] = neg ? (int32_t)(0u - (uint32_t)v->coefsT[src]) : v->coefsT[src];
        }
        acc[0].current_variance = 3.25;
        tfhe_blindRotate_FFT(&acc[0], ck->bkFFT->bkFFT, bara, n, gp);
        check("blindRotate_FFT keeps the accumulator's variance", acc[0].current_variance == 3.25);
        int ok = acc[0].b->coefsT[0] == u[0].b;
        for (int32_t c = 0; c < k; c++)
            for (int32_t j = 0; j < N; j++) {
                const int32_t want = j == 0 ? acc[0].a[c].coefsT[0] : (int32_t)(0u - (uint32_t)acc[0].a[c].coefsT[N - j]);
                ok &= u[0].a[c * N + j] == want;
            }
        check("blindRotate_FFT + extraction == bootstrap_woKS_FFT", ok);

        /* bootstrap with keyswitch, and lweKeySwitch of the extracted sample */
        tfhe_bootstrap_FFT(&y[0], ck->bkFFT, mu, &x[0]);
        put_lwe(rec, &y[0], n);
        put_f64(rec, y[0].current_variance);
        lweKeySwitch(&y[1], ck->bkFFT->ks, &u[0]);
        put_lwe(rec, &y[1], n);
        put_f64(rec, y[1].current_variance);
        check("lweKeySwitch(woKS) == bootstrap_FFT", same_lwe(&y[1], &y[0], n) &&
                                                        y[1].current_variance == y[0].current_variance);
        tfhe_bootstrap(&y[2], ck->bk, mu, &x[0]);
        check("tfhe_bootstrap == tfhe_bootstrap_FFT", same_lwe(&y[2], &y[0], n) &&
                                                         y[2].current_variance == y[0].current_variance);

        /* a NAND gate and the extracted sample it keyswitches: (0,1/8) - x0 - x1 bootstrapped */
        bootsNAND(&y[3], &x[0], &x[1], ck);
        lweNoiselessTrivial(comb, modSwitchToTorus32(1, 8), io);
        lweSubTo(comb, &x[0], io);
        lweSubTo(comb, &x[1], io);
        tfhe_bootstrap_woKS_FFT(&u[2], ck->bkFFT, mu, comb);
        put_lwe(rec, &u[2], kN);
        put_lwe(rec, &y[3], n);
        put_f64(rec, y[3].current_variance);
        check("NAND decrypts", bootsSymDecrypt(&y[3], key) == 1 - (bit0 & bit1));

        /* coefficient-domain rotation on the keyset's own samples and on a caller-made copy */
        const int32_t first = 100 + 37 * t, steps = 3;
        for (int32_t j = 0; j < N; j++)
            for (int32_t c = 0; c <= k; c++) acc[1].a[c].coefsT[j] = (int32_t)next32();
        copy_tlwe(&acc[2], &acc[1], k, N);
        copy_tlwe(&acc[3], &acc[1], k, N);
        tfhe_blindRotate_FFT(&acc[1], ck->bkFFT->bkFFT + first, bara, steps, gp);
        tfhe_blindRotate(&acc[2], ck->bk->bk + first, bara, steps, gp);
        check("blindRotate (own samples) == blindRotate_FFT", same_tlwe(&acc[2], &acc[1], k, N));
        TGswSample *copy = (TGswSample *)malloc(sizeof(TGswSample) * (size_t)steps);
        TLweSample *rows = new_TLweSample_array(steps * kpl, tp);
        TLweSample **blocs = (TLweSample **)malloc(sizeof(TLweSample *) * (size_t)steps * (size_t)(k + 1));
        for (int32_t s = 0; s < steps; s++) {
            for (int32_t r = 0; r < kpl; r++) copy_tlwe(&rows[s * kpl + r], &ck->bk->bk[first + s].all_sample[r], k, N);
            for (int32_t c = 0; c <= k; c++) blocs[s * (k + 1) + c] = &rows[s * kpl + c * l];
            TGswSample g = {&rows[s * kpl], &blocs[s * (k + 1)], k, l};
            memcpy(&copy[s], &g, sizeof g);
        }
        tfhe_blindRotate(&acc[3], copy, bara, steps, gp);
        check("blindRotate (caller-made samples) == blindRotate_FFT", same_tlwe(&acc[3], &acc[1], k, N));

        /* 5 samples at once == 2 then 3 */
        copy_tlwe(&acc[2], &acc[1], k, N);
        tfhe_blindRotate_FFT(&acc[1], ck->bkFFT->bkFFT + 10, bara + 20, 5, gp);
        tfhe_blindRotate_FFT(&acc[2], ck->bkFFT->bkFFT + 10, bara + 20, 2, gp);
        tfhe_blindRotate_FFT(&acc[2], ck->bkFFT->bkFFT + 12, bara + 22, 3, gp);
        check("rotation over 5 samples == over 2 then 3", same_tlwe(&acc[2], &acc[1], k, N));

        /* one CMUX step from the external product: acc + bk_i (x) ((X^a - 1) acc) */
        const int32_t i = (int32_t)(next32() % (uint32_t)n), a = 1 + (int32_t)(next32() % (uint32_t)(2 * N - 1));
        for (int32_t c = 0; c <= k; c++)
            for (int32_t j = 0; j < N; j++) {
                /* (X^a - 1) * poly: coefficient j is +-poly[(j - a) mod N] - poly[j] */
                int32_t src = j - a, neg = 0;
                while (src < 0) {
                    src += N;
                    neg ^= 1;
                }
                const uint32_t r = neg ? 0u - (uint32_t)acc[1].a[c].coefsT[src] : (uint32_t)acc[1].a[c].coefsT[src];
                acc[2].a[c].coefsT[j] = (int32_t)(r - (uint32_t)acc[1].a[c].coefsT[j]);
            }
        acc[2].current_variance = 0.75;
        tGswExternProduct(&acc[3], &ck->bk->bk[i], &acc[2], gp);
        put_i32(rec, &i, 1);
        put_tlwe(rec, &acc[2], k, N);
        put_f64(rec, acc[2].current_variance);
        put_tlwe(rec, &acc[3], k, N);
        put_f64(rec, acc[3].current_variance);
        const double prod_var = acc[3].current_variance;
        for (int32_t c = 0; c <= k; c++)
            for (int32_t j = 0; j < N; j++)
                acc[3].a[c].coefsT[j] = (int32_t)((uint32_t)acc[3].a[c].coefsT[j] + (uint32_t)acc[1].a[c].coefsT[j]);
        tfhe_blindRotate_FFT(&acc[1], ck->bkFFT->bkFFT + i, &a, 1, gp);
        check("acc + tGswExternProduct == one CMUX step", same_tlwe(&acc[3], &acc[1], k, N));
        /* tGswExternMulToTLwe: the same product in place, without b's variance */
        copy_tlwe(&acc[0], &acc[2], k, N);
        tGswExternProduct(&acc[3], &ck->bk->bk[i], &acc[2], gp);
        tGswExternMulToTLwe(&acc[0], &ck->bk->bk[i], gp);
        check("tGswExternMulToTLwe == tGswExternProduct", same_tlwe(&acc[0], &acc[3], k, N));
        check("tGswExternMulToTLwe leaves out b's variance", acc[0].current_variance + 0.75 == prod_var);

        free(copy);
        free(blocs);
        delete_TLweSample_array(steps * kpl, rows);
    }
    fclose(rec);
    free(bara);
    delete_TorusPolynomial(v);
    delete_TLweSample_array(4, acc);
    delete_LweSample_array(4, u);
    delete_LweSample(comb);
    delete_LweSample_array(4, y);
    delete_LweSample_array(2, x);
    delete_gate_bootstrapping_secret_keyset(key);
    if (fails) return 1;
    printf("OK\n");
    return 0;
}
