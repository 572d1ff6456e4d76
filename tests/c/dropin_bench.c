/* Throughput of the drop-in gate API as a reference user calls it: one bootsNAND at a time, from T
 * threads at once on one cloud keyset (each thread its own operands and results).  Prints one JSON
 * object: threads, gates, seconds (wall time from the common start to the last thread's end),
 * gates_per_s and the number of results that do not decrypt to the truth table.
 *
 *   dropin_bench <precision 0|1> <threads> <gates per thread> */
#include <pthread.h>
#include <stdio.h>
#include <stdlib.h>
#include <time.h>

#include "tfhe.h"

static const TFheGateBootstrappingSecretKeySet *key;
static pthread_barrier_t start;
static int per_thread;

struct work {
    LweSample *a, *b, *r;
    int *va, *vb;
    int errors;
};

static double now(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + 1e-9 * ts.tv_nsec;
}

static void *run(void *arg) {
    struct work *w = (struct work *)arg;
    pthread_barrier_wait(&start);
    for (int i = 0; i < per_thread; i++) bootsNAND(&w->r[i], &w->a[i], &w->b[i], &key->cloud);
    return NULL;
}

int main(int argc, char **argv) {
    if (argc < 4) return 2;
    tfhe_b200_set_precision(atoi(argv[1]));
    const int threads = atoi(argv[2]);
    per_thread = atoi(argv[3]);
    uint32_t seed[] = {5, 6, 7};
    tfhe_random_generator_setSeed(seed, 3);
    TFheGateBootstrappingParameterSet *params = new_default_gate_bootstrapping_parameters(110);
    TFheGateBootstrappingSecretKeySet *k = new_random_gate_bootstrapping_secret_keyset(params);
    key = k;
    struct work *w = calloc(threads, sizeof *w);
    pthread_t *th = calloc(threads, sizeof *th);
    for (int t = 0; t < threads; t++) {
        w[t].a = new_gate_bootstrapping_ciphertext_array(per_thread, params);
        w[t].b = new_gate_bootstrapping_ciphertext_array(per_thread, params);
        w[t].r = new_gate_bootstrapping_ciphertext_array(per_thread, params);
        w[t].va = malloc(per_thread * sizeof(int));
        w[t].vb = malloc(per_thread * sizeof(int));
        for (int i = 0; i < per_thread; i++) {
            w[t].va[i] = rand() & 1;
            w[t].vb[i] = rand() & 1;
            bootsSymEncrypt(&w[t].a[i], w[t].va[i], key);
            bootsSymEncrypt(&w[t].b[i], w[t].vb[i], key);
        }
    }
    /* one gate first, so that moving the key to the GPU is not timed */
    bootsNAND(&w[0].r[0], &w[0].a[0], &w[0].b[0], &key->cloud);
    pthread_barrier_init(&start, NULL, threads + 1);
    for (int t = 0; t < threads; t++) pthread_create(&th[t], NULL, run, &w[t]);
    pthread_barrier_wait(&start);
    const double t0 = now();
    for (int t = 0; t < threads; t++) pthread_join(th[t], NULL);
    const double sec = now() - t0;
    int errors = 0;
    for (int t = 0; t < threads; t++)
        for (int i = 0; i < per_thread; i++)
            errors += bootsSymDecrypt(&w[t].r[i], key) != !(w[t].va[i] & w[t].vb[i]);
    const long gates = (long)threads * per_thread;
    printf("{\"threads\": %d, \"gates\": %ld, \"seconds\": %.6f, \"gates_per_s\": %.1f, \"errors\": %d}\n", threads, gates,
           sec, gates / sec, errors);
    return errors ? 1 : 0;
}
