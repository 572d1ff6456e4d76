/* A client program for the reference's file API (tfhe_io.h, gate-bootstrapping part), compiled as
 * plain C against include/tfhe.h and linked with libtfhe_b200.so.  No GPU is needed: it only moves
 * keys and ciphertexts through files and decrypts on the host.
 *
 *   dropin_io KEYSET CTS COUNT OUT_KEYSET OUT_CTS OUT_PARAMS
 *
 * reads a secret key set and COUNT ciphertexts written by the reference, prints the decrypted
 * bits on one line, and writes the key set, the ciphertexts and the parameter set back with the
 * export functions (the caller compares the files byte for byte). */
#include <stdio.h>
#include <stdlib.h>

#include "tfhe.h"

int main(int argc, char **argv) {
    if (argc != 7) return 2;
    const int count = atoi(argv[3]);

    FILE *f = fopen(argv[1], "rb");
    if (!f) return 3;
    TFheGateBootstrappingSecretKeySet *key = new_tfheGateBootstrappingSecretKeySet_fromFile(f);
    fclose(f);
    const TFheGateBootstrappingParameterSet *params = key->params;

    LweSample *cts = new_gate_bootstrapping_ciphertext_array(count, params);
    f = fopen(argv[2], "rb");
    if (!f) return 4;
    for (int i = 0; i < count; i++) import_gate_bootstrapping_ciphertext_fromFile(f, &cts[i], params);
    fclose(f);
    for (int i = 0; i < count; i++) printf("%d", bootsSymDecrypt(&cts[i], key));
    printf("\n");

    f = fopen(argv[4], "wb");
    export_tfheGateBootstrappingSecretKeySet_toFile(f, key);
    fclose(f);
    f = fopen(argv[5], "wb");
    for (int i = 0; i < count; i++) export_gate_bootstrapping_ciphertext_toFile(f, &cts[i], params);
    fclose(f);
    f = fopen(argv[6], "wb");
    export_tfheGateBootstrappingParameterSet_toFile(f, params);
    fclose(f);

    /* the cloud part alone, read back through the cloud-keyset reader */
    f = tmpfile();
    export_tfheGateBootstrappingCloudKeySet_toFile(f, &key->cloud);
    rewind(f);
    TFheGateBootstrappingCloudKeySet *cloud = new_tfheGateBootstrappingCloudKeySet_fromFile(f);
    fclose(f);
    if (cloud->params->in_out_params->n != params->in_out_params->n) return 5;
    delete_gate_bootstrapping_cloud_keyset(cloud);

    delete_gate_bootstrapping_ciphertext_array(count, cts);
    delete_gate_bootstrapping_secret_keyset(key);
    return 0;
}
