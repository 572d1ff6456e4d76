// multi.cu -- one batch of gates sharded across several cloud keys, each resident on its own GPU.
//
// Gate bootstrapping has no exchange between gates of one batch: every gate reads its own input
// ciphertexts and the (replicated) cloud key.  Multi-GPU throughput is therefore replica sharding:
// the batch is cut into contiguous shards, shard k runs on key k (tfheb_gate_batch on that key's
// device and stream) in its own host thread, and the shards write disjoint rows of the output.
// There is no collective.  Results are bit-identical to one tfheb_gate_batch over the whole batch,
// since every kernel of the path is deterministic per gate.
#include <string>
#include <thread>
#include <vector>

#include "internal.h"

using namespace tfheb;

extern "C" {

tfheb_status tfheb_gate_batch_multi(tfheb_cloud_key *const *cks, int32_t nkeys, int32_t gate, int32_t precision,
                                    int32_t count, const int32_t *a, const int32_t *b, const int32_t *c,
                                    int32_t *out) {
    if (!cks || nkeys < 1 || count < 0 || (count > 0 && (!a || !out))) {
        set_error("tfheb_gate_batch_multi: invalid arguments");
        return TFHEB_ERR_INVALID;
    }
    for (int32_t k = 0; k < nkeys; k++) {
        if (!cks[k]) {
            set_error("tfheb_gate_batch_multi: key " + std::to_string(k) + " is NULL");
            return TFHEB_ERR_INVALID;
        }
        const tfheb_params &p0 = cks[0]->ck.p, &pk = cks[k]->ck.p;
        if (pk.n != p0.n || pk.N != p0.N || pk.k != p0.k || pk.l != p0.l || pk.Bgbit != p0.Bgbit ||
            pk.ks_t != p0.ks_t || pk.ks_basebit != p0.ks_basebit) {
            set_error("tfheb_gate_batch_multi: key " + std::to_string(k) + " has another parameter set than key 0");
            return TFHEB_ERR_INVALID;
        }
    }
    if (count == 0) return TFHEB_OK;
    const size_t row = (size_t)cks[0]->ck.p.n + 1;
    auto lo = [&](int32_t k) { return (int32_t)((int64_t)count * k / nkeys); };
    std::vector<tfheb_status> st(nkeys, TFHEB_OK);
    std::vector<std::string> msg(nkeys);
    auto shard = [&](int32_t k) {
        const int32_t first = lo(k), n = lo(k + 1) - first;
        if (n == 0) return;
        const size_t off = (size_t)first * row;
        st[k] = tfheb_gate_batch(cks[k], gate, precision, n, a + off, b ? b + off : nullptr, c ? c + off : nullptr,
                                 out + off);
        if (st[k] != TFHEB_OK) msg[k] = tfheb_last_error();  // the message is per thread
    };
    if (nkeys == 1) {
        shard(0);
    } else {
        std::vector<std::thread> workers;
        workers.reserve(nkeys);
        for (int32_t k = 0; k < nkeys; k++) workers.emplace_back(shard, k);
        for (auto &w : workers) w.join();
    }
    for (int32_t k = 0; k < nkeys; k++)
        if (st[k] != TFHEB_OK) {
            set_error("tfheb_gate_batch_multi: shard " + std::to_string(k) + ": " + msg[k]);
            return st[k];
        }
    return TFHEB_OK;
}

}  // extern "C"
