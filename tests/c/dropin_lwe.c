/* A client of the reference's LWE helpers and coefficient-domain bootstrap (lwe-functions.h,
 * tfhe.h:38-39), compiled as plain C against include/tfhe.h and linked with libtfhe_b200.so.
 *
 *   dropin_lwe host   LWE encryption, decryption and arithmetic on the host (no GPU needed)
 *   dropin_lwe gpu    tfhe_bootstrap / tfhe_bootstrap_woKS on the GPU
 *
 * Exit status 0 when every check holds; a failing check prints its name. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "tfhe.h"

static int fails = 0;
static void check(const char *name, long long got, long long want) {
    if (got != want) {
        fprintf(stderr, "%s: got %lld want %lld\n", name, got, want);
        fails++;
    }
}

int main(int argc, char **argv) {
    const int gpu = argc > 1 && strcmp(argv[1], "gpu") == 0;
    uint32_t seed[] = {7, 11};
    tfhe_random_generator_setSeed(seed, 2);
    TFheGateBootstrappingParameterSet *params = new_default_gate_bootstrapping_parameters(110);
    TFheGateBootstrappingSecretKeySet *key = new_random_gate_bootstrapping_secret_keyset(params);
    const LweParams *io = params->in_out_params;
    const LweKey *lk = key->lwe_key;
    const double alpha = io->alpha_min;
    LweSample *x = new_gate_bootstrapping_ciphertext_array(4, params);

    if (!gpu) {
        /* messages of the 8-slot torus decrypt exactly */
        for (int m = -4; m < 4; m++) {
            const Torus32 mu = modSwitchToTorus32(m, 8);
            lweSymEncrypt(&x[0], mu, alpha, lk);
            check("lweSymDecrypt", lweSymDecrypt(&x[0], lk, 8), mu);
        }
        check("variance", x[0].current_variance == alpha * alpha, 1);
        /* (3/8) + (1/8) = 1/2, (3/8) - 2 * (1/8) = 1/8, -(3/8) */
        lweSymEncrypt(&x[0], modSwitchToTorus32(3, 8), alpha, lk);
        lweSymEncrypt(&x[1], modSwitchToTorus32(1, 8), alpha, lk);
        lweCopy(&x[2], &x[0], io);
        lweAddTo(&x[2], &x[1], io);
        check("lweAddTo", lweSymDecrypt(&x[2], lk, 8), modSwitchToTorus32(4, 8));
        check("lweAddTo variance", x[2].current_variance == 2 * alpha * alpha, 1);
        lweCopy(&x[2], &x[0], io);
        lweSubMulTo(&x[2], 2, &x[1], io);
        check("lweSubMulTo", lweSymDecrypt(&x[2], lk, 8), modSwitchToTorus32(1, 8));
        check("lweSubMulTo variance", x[2].current_variance == 5 * alpha * alpha, 1);
        lweCopy(&x[2], &x[0], io);
        lweAddMulTo(&x[2], 3, &x[1], io);
        check("lweAddMulTo", lweSymDecrypt(&x[2], lk, 8), modSwitchToTorus32(6, 8));
        lweCopy(&x[2], &x[0], io);
        lweSubTo(&x[2], &x[1], io);
        check("lweSubTo", lweSymDecrypt(&x[2], lk, 8), modSwitchToTorus32(2, 8));
        lweNegate(&x[2], &x[0], io);
        check("lweNegate", lweSymDecrypt(&x[2], lk, 8), modSwitchToTorus32(-3, 8));
        lweNoiselessTrivial(&x[2], modSwitchToTorus32(5, 16), io);
        check("lweNoiselessTrivial", lwePhase(&x[2], lk), modSwitchToTorus32(5, 16));
        lweClear(&x[2], io);
        check("lweClear", lwePhase(&x[2], lk), 0);
        /* external noise lands in the phase exactly: dtot32(1/64) = 2^26 */
        lweSymEncryptWithExternalNoise(&x[3], modSwitchToTorus32(1, 4), 1.0 / 64, alpha, lk);
        check("lweSymEncryptWithExternalNoise", lwePhase(&x[3], lk), modSwitchToTorus32(1, 4) + (1 << 26));
    } else {
        const Torus32 mu = modSwitchToTorus32(1, 8);
        for (int bit = 0; bit < 2; bit++) {
            bootsSymEncrypt(&x[0], bit, key);
            tfhe_bootstrap(&x[1], key->cloud.bk, mu, &x[0]);
            check("tfhe_bootstrap", bootsSymDecrypt(&x[1], key), bit);
            tfhe_bootstrap_FFT(&x[2], key->cloud.bkFFT, mu, &x[0]);
            check("tfhe_bootstrap == tfhe_bootstrap_FFT", memcmp(x[1].a, x[2].a, sizeof(Torus32) * io->n) == 0 &&
                                                              x[1].b == x[2].b, 1);
            /* without keyswitch: samples of the extracted dimension k*N */
            const int kN = params->tgsw_params->tlwe_params->N * params->tgsw_params->tlwe_params->k;
            LweSample u = {calloc(kN, sizeof(Torus32)), 0, 0.}, v = {calloc(kN, sizeof(Torus32)), 0, 0.};
            tfhe_bootstrap_woKS(&u, key->cloud.bk, mu, &x[0]);
            tfhe_bootstrap_woKS_FFT(&v, key->cloud.bkFFT, mu, &x[0]);
            check("tfhe_bootstrap_woKS == tfhe_bootstrap_woKS_FFT",
                  memcmp(u.a, v.a, sizeof(Torus32) * kN) == 0 && u.b == v.b, 1);
            free(u.a);
            free(v.a);
        }
    }
    delete_gate_bootstrapping_ciphertext_array(4, x);
    delete_gate_bootstrapping_secret_keyset(key);
    delete_gate_bootstrapping_parameters(params);
    return fails ? 1 : 0;
}
