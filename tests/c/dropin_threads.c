/* Concurrent callers of the drop-in gate API: several POSIX threads evaluate gates with one cloud
 * keyset at the same time, starting together on a keyset whose key is not yet on the GPU, as a
 * multithreaded reference user would (the reference's gates are reentrant across threads on
 * distinct outputs: fft_processor_spqlios.cpp:123).  Each thread also overwrites one of its inputs
 * with a gate result (result aliasing an operand, as test-long-run.cpp does).  Exit status 0 when
 * every result decrypts to its truth table. */
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>

#include "tfhe.h"

enum { THREADS = 4, GATES = 6 };

static const TFheGateBootstrappingParameterSet *params;
static const TFheGateBootstrappingSecretKeySet *key;
static pthread_barrier_t start;

struct work {
    LweSample *a, *b, *r;
    int va[GATES], vb[GATES], fails;
};

static void *run(void *arg) {
    struct work *w = (struct work *)arg;
    const TFheGateBootstrappingCloudKeySet *ck = &key->cloud;
    pthread_barrier_wait(&start);
    for (int i = 0; i < GATES; i++) bootsNAND(&w->r[i], &w->a[i], &w->b[i], ck);
    for (int i = 0; i < GATES; i++)
        if (bootsSymDecrypt(&w->r[i], key) != !(w->va[i] & w->vb[i])) w->fails++;
    bootsXOR(&w->a[0], &w->a[0], &w->b[0], ck); /* result aliases an operand */
    if (bootsSymDecrypt(&w->a[0], key) != (w->va[0] ^ w->vb[0])) w->fails++;
    bootsMUX(&w->b[1], &w->a[1], &w->b[1], &w->r[1], ck);
    if (bootsSymDecrypt(&w->b[1], key) != (w->va[1] ? w->vb[1] : !(w->va[1] & w->vb[1]))) w->fails++;
    return NULL;
}

int main(int argc, char **argv) {
    tfhe_b200_set_precision(argc > 1 ? atoi(argv[1]) : 0);
    uint32_t seed[] = {11, 22, 33};
    tfhe_random_generator_setSeed(seed, 3);
    TFheGateBootstrappingParameterSet *p = new_default_gate_bootstrapping_parameters(110);
    TFheGateBootstrappingSecretKeySet *k = new_random_gate_bootstrapping_secret_keyset(p);
    params = p;
    key = k;
    struct work w[THREADS];
    pthread_t th[THREADS];
    pthread_barrier_init(&start, NULL, THREADS);
    for (int t = 0; t < THREADS; t++) {
        w[t].a = new_gate_bootstrapping_ciphertext_array(GATES, params);
        w[t].b = new_gate_bootstrapping_ciphertext_array(GATES, params);
        w[t].r = new_gate_bootstrapping_ciphertext_array(GATES, params);
        w[t].fails = 0;
        for (int i = 0; i < GATES; i++) {
            w[t].va[i] = (i + t) & 1;
            w[t].vb[i] = ((i + t) >> 1) & 1;
            bootsSymEncrypt(&w[t].a[i], w[t].va[i], key);
            bootsSymEncrypt(&w[t].b[i], w[t].vb[i], key);
        }
    }
    for (int t = 0; t < THREADS; t++) pthread_create(&th[t], NULL, run, &w[t]);
    int fails = 0;
    for (int t = 0; t < THREADS; t++) {
        pthread_join(th[t], NULL);
        fails += w[t].fails;
        delete_gate_bootstrapping_ciphertext_array(GATES, w[t].a);
        delete_gate_bootstrapping_ciphertext_array(GATES, w[t].b);
        delete_gate_bootstrapping_ciphertext_array(GATES, w[t].r);
    }
    pthread_barrier_destroy(&start);
    delete_gate_bootstrapping_secret_keyset(k);
    delete_gate_bootstrapping_parameters(p);
    printf("%s\n", fails ? "FAIL" : "OK");
    return fails ? 1 : 0;
}
