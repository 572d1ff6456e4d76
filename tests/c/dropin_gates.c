/* A client program written against the reference's gate-bootstrapping API (the calling pattern of
 * the reference's test-gate-bootstrapping.cpp and test-c-binding.c), compiled as plain C against
 * include/tfhe.h and linked with libtfhe_b200.so.  Exit status 0 when every gate decrypts to its
 * truth table. */
#include <stdio.h>
#include <stdlib.h>

#include "tfhe.h"

static int check(const char *name, int got, int want, int *fails) {
    if (got != want) {
        fprintf(stderr, "%s: got %d want %d\n", name, got, want);
        (*fails)++;
    }
    return got;
}

int main(int argc, char **argv) {
    int precision = argc > 1 ? atoi(argv[1]) : 0;
    const int lambda = argc > 2 ? atoi(argv[2]) : 110;  /* <= 80: the reference's 80-bit set */
    uint32_t seed[] = {314, 42, 2024};
    tfhe_random_generator_setSeed(seed, 3);
    tfhe_b200_set_precision(precision);

    TFheGateBootstrappingParameterSet *params = new_default_gate_bootstrapping_parameters(lambda);
    TFheGateBootstrappingSecretKeySet *key = new_random_gate_bootstrapping_secret_keyset(params);
    const TFheGateBootstrappingCloudKeySet *ck = &key->cloud;
    if (params->in_out_params->n != (lambda <= 80 ? 500 : 630) || params->tgsw_params->tlwe_params->N != 1024) return 2;

    enum { NB = 8 };
    LweSample *a = new_gate_bootstrapping_ciphertext_array(NB, params);
    LweSample *b = new_gate_bootstrapping_ciphertext_array(NB, params);
    LweSample *c = new_gate_bootstrapping_ciphertext_array(NB, params);
    LweSample *r = new_gate_bootstrapping_ciphertext_array(NB, params);
    int va[NB], vb[NB], vc[NB], fails = 0;
    for (int i = 0; i < NB; i++) {
        va[i] = i & 1;
        vb[i] = (i >> 1) & 1;
        vc[i] = (i >> 2) & 1;
        bootsSymEncrypt(&a[i], va[i], key);
        bootsSymEncrypt(&b[i], vb[i], key);
        bootsSymEncrypt(&c[i], vc[i], key);
    }
    for (int i = 0; i < NB; i++) {
        bootsNAND(&r[i], &a[i], &b[i], ck);
        check("NAND", bootsSymDecrypt(&r[i], key), !(va[i] && vb[i]), &fails);
        bootsXOR(&r[i], &a[i], &b[i], ck);
        check("XOR", bootsSymDecrypt(&r[i], key), va[i] ^ vb[i], &fails);
        bootsORYN(&r[i], &a[i], &b[i], ck);
        check("ORYN", bootsSymDecrypt(&r[i], key), va[i] || !vb[i], &fails);
        bootsMUX(&r[i], &a[i], &b[i], &c[i], ck);
        check("MUX", bootsSymDecrypt(&r[i], key), va[i] ? vb[i] : vc[i], &fails);
        bootsNOT(&r[i], &a[i], ck);
        check("NOT", bootsSymDecrypt(&r[i], key), !va[i], &fails);
        bootsCONSTANT(&r[i], vb[i], ck);
        check("CONSTANT", bootsSymDecrypt(&r[i], key), vb[i], &fails);
        /* the output may alias an input */
        bootsCOPY(&r[i], &a[i], ck);
        bootsAND(&r[i], &r[i], &b[i], ck);
        check("AND (aliased)", bootsSymDecrypt(&r[i], key), va[i] && vb[i], &fails);
    }
    /* batched extension over reference-style arrays */
    bootsNAND_batch(r, a, b, NB, ck);
    for (int i = 0; i < NB; i++) check("NAND_batch", bootsSymDecrypt(&r[i], key), !(va[i] && vb[i]), &fails);
    /* a 3-level NAND tree: (a NAND b) NAND (b NAND c) */
    LweSample *t1 = new_gate_bootstrapping_ciphertext(params), *t2 = new_gate_bootstrapping_ciphertext(params);
    for (int i = 0; i < NB; i++) {
        bootsNAND(t1, &a[i], &b[i], ck);
        bootsNAND(t2, &b[i], &c[i], ck);
        bootsNAND(&r[i], t1, t2, ck);
        check("tree", bootsSymDecrypt(&r[i], key), !(!(va[i] && vb[i]) && !(vb[i] && vc[i])), &fails);
    }
    delete_gate_bootstrapping_ciphertext(t2);
    delete_gate_bootstrapping_ciphertext(t1);
    delete_gate_bootstrapping_ciphertext_array(NB, r);
    delete_gate_bootstrapping_ciphertext_array(NB, c);
    delete_gate_bootstrapping_ciphertext_array(NB, b);
    delete_gate_bootstrapping_ciphertext_array(NB, a);
    delete_gate_bootstrapping_secret_keyset(key);
    delete_gate_bootstrapping_parameters(params);
    printf("%s\n", fails ? "FAIL" : "OK");
    return fails ? 1 : 0;
}
