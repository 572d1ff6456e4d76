// dropin.cu -- the reference's gate-bootstrapping C API (include/tfhe.h) on top of the engine.
//
// Same symbols and caller-visible struct layouts as tfhe v1.1 (tfhe_gate_bootstrapping_functions.h,
// tfhe_gate_bootstrapping_structures.h); errors keep the reference's convention of void functions
// that abort on a fatal condition (tfhe_gate_bootstrapping.cpp:11-15 die_dramatically).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <vector>

#include "../../include/tfhe.h"
#include "internal.h"

struct TGswKey {
    tfheb_secret_key *sk;
};
struct LweBootstrappingKey {
    tfheb_cloud_key *ck;
};
// One single-gate call waiting to be evaluated (see run_combined).
struct GateRequest {
    int32_t gate;
    LweSample *res;
    const LweSample *a, *b, *c;
    bool done;
};

struct LweBootstrappingKeyFFT {
    LweBootstrappingKeyFFT(tfheb_cloud_key *key, int32_t lwe_n, int32_t ext_n) : ck(key), n(lwe_n), kN(ext_n) {}
    tfheb_cloud_key *ck;
    int32_t n, kN;
    std::atomic<int32_t> on_device_mask{0};  // precisions whose FFT-domain key is on the device
    // single-gate calls from concurrent threads, combined into batches
    std::mutex comb_mu;
    std::condition_variable comb_cv;      // callers waiting for their results or their turn
    std::condition_variable comb_arrive;  // the batch's leader gathering requests
    std::vector<GateRequest *> comb_pending;
    bool comb_busy = false;
    size_t comb_last = 0;  // requests in the previous batch
};

namespace {

[[noreturn]] void die(const char *what) {
    std::fprintf(stderr, "tfhe_b200: %s: %s\n", what, tfheb_last_error());
    std::abort();
}

std::mutex g_rng_mu;
uint64_t g_rng_state = 0x243F6A8885A308D3ull;  // reseeded by tfhe_random_generator_setSeed
std::atomic<int32_t> g_precision{TFHEB_FP64};  // set by tfhe_b200_set_precision, read by every gate

uint64_t next_seed() {
    std::lock_guard<std::mutex> lock(g_rng_mu);
    uint64_t z = (g_rng_state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

int device_index() {
    const char *e = std::getenv("TFHE_B200_DEVICE");
    return e ? std::atoi(e) : 0;
}

tfheb_params to_params(const TFheGateBootstrappingParameterSet *ps) {
    const TLweParams *tp = ps->tgsw_params->tlwe_params;
    return tfheb_params{ps->in_out_params->n, tp->N, tp->k, ps->tgsw_params->l, ps->tgsw_params->Bgbit,
                        ps->ks_t, ps->ks_basebit, ps->in_out_params->alpha_min, tp->alpha_min};
}

template <typename T>
T *make(const T &v) {  // objects with const members: construct once, copy bytes
    T *p = static_cast<T *>(std::malloc(sizeof(T)));
    std::memcpy(static_cast<void *>(p), &v, sizeof(T));
    return p;
}

TFheGateBootstrappingParameterSet *make_params(const tfheb_params &p, double in_alpha_max, double tlwe_alpha_max) {
    LweParams *in = make(LweParams{p.n, p.ks_stdev, in_alpha_max});
    TLweParams *acc = make(TLweParams{p.N, p.k, p.bk_stdev, tlwe_alpha_max,
                                      LweParams{p.k * p.N, p.bk_stdev, tlwe_alpha_max}});
    Torus32 *h = static_cast<Torus32 *>(std::malloc(sizeof(Torus32) * p.l));
    uint32_t sum = 0;
    for (int i = 0; i < p.l; i++) {
        h[i] = (Torus32)(1u << (32 - (i + 1) * p.Bgbit));
        sum += 1u << (32 - (i + 1) * p.Bgbit);
    }
    const int32_t Bg = 1 << p.Bgbit;
    TGswParams *gp = make(TGswParams{p.l, p.Bgbit, Bg, Bg / 2, (uint32_t)(Bg - 1), acc, (p.k + 1) * p.l, h,
                                     sum * (uint32_t)(Bg / 2)});
    return make(TFheGateBootstrappingParameterSet{p.ks_t, p.ks_basebit, in, gp});
}

// The drop-in objects around an engine key pair (the keysets own sk and ck).
TFheGateBootstrappingCloudKeySet assemble_cloud(const TFheGateBootstrappingParameterSet *params, tfheb_cloud_key *ck) {
    const tfheb_params p = to_params(params);
    return TFheGateBootstrappingCloudKeySet{params, new LweBootstrappingKey{ck},
                                            new LweBootstrappingKeyFFT(ck, p.n, p.k * p.N)};
}
TFheGateBootstrappingSecretKeySet *assemble_secret_keyset(const TFheGateBootstrappingParameterSet *params,
                                                          tfheb_secret_key *sk, tfheb_cloud_key *ck) {
    const int32_t n = params->in_out_params->n;
    int32_t *key = static_cast<int32_t *>(std::malloc(sizeof(int32_t) * n));
    tfheb_secret_key_export(sk, key, nullptr);
    LweKey *lk = make(LweKey{params->in_out_params, key});
    return make(TFheGateBootstrappingSecretKeySet{params, lk, new TGswKey{sk}, assemble_cloud(params, ck)});
}

// Moves the key of the current precision to the device on first use.  Threads may race here on a
// fresh keyset: the transfer runs under the key's own lock and skips a precision already present,
// so a second caller only waits; the mask is atomic.
void ensure_on_device(LweBootstrappingKeyFFT *f) {
    const int32_t bit = 1 << g_precision;
    if (f->on_device_mask.load(std::memory_order_acquire) & bit) return;
    if (tfheb_cloud_key_to_device(f->ck, device_index(), bit, 0) != TFHEB_OK) die("moving the key to the GPU");
    f->on_device_mask.fetch_or(bit, std::memory_order_release);
}

LweBootstrappingKeyFFT *ready(const TFheGateBootstrappingCloudKeySet *bk) {
    auto *f = const_cast<LweBootstrappingKeyFFT *>(bk->bkFFT);
    if (!f || !f->ck) die("cloud keyset has no key");
    ensure_on_device(f);
    return f;
}

// Evaluates a set of single-gate requests: one batch per gate code present.  Every request's
// operands are copied before its group's results are written, so a result may alias its own operands.
void evaluate_requests(LweBootstrappingKeyFFT *f, const std::vector<GateRequest *> &reqs) {
    const int32_t n = f->n, row = n + 1;
    for (int32_t code = 0; code < TFHEB_NOT; code++) {
        std::vector<GateRequest *> grp;
        for (GateRequest *r : reqs)
            if (r->gate == code) grp.push_back(r);
        if (grp.empty()) continue;
        const size_t cnt = grp.size();
        std::vector<int32_t> ha(cnt * row), hb(cnt * row), hc(code == TFHEB_MUX ? cnt * row : 0), out(cnt * row);
        auto put = [&](std::vector<int32_t> &buf, size_t i, const LweSample *x) {
            std::memcpy(&buf[i * row], x->a, sizeof(int32_t) * n);
            buf[i * row + n] = x->b;
        };
        for (size_t i = 0; i < cnt; i++) {
            put(ha, i, grp[i]->a);
            put(hb, i, grp[i]->b);
            if (code == TFHEB_MUX) put(hc, i, grp[i]->c);
        }
        if (tfheb_gate_batch(f->ck, code, g_precision, (int32_t)cnt, ha.data(), hb.data(),
                             code == TFHEB_MUX ? hc.data() : nullptr, out.data()) != TFHEB_OK)
            die("gate evaluation");
        for (size_t i = 0; i < cnt; i++) {
            std::memcpy(grp[i]->res->a, &out[i * row], sizeof(int32_t) * n);
            grp[i]->res->b = out[i * row + n];
            grp[i]->res->current_variance = 0.;
        }
    }
}

// Longest time a batch's leader waits for the callers of the previous batch to post their next
// gates: about 5 % of one single-bootstrap launch.
constexpr auto kGatherWait = std::chrono::microseconds(200);

// One bootstrapped gate from one caller.  Calls from concurrent threads are combined: a caller
// queues its request, and whichever caller finds no evaluation running becomes the leader: it takes
// every queued request and evaluates them together (one batch per gate code, evaluate_requests)
// while the others wait; when it is done, a caller whose request arrived meanwhile leads the next
// batch.  Callers that just got their results need a moment to post their next gates, so a leader
// with fewer requests than the previous batch had waits up to kGatherWait for them.  A lone caller
// evaluates its own gate at once; N concurrent callers share one launch sequence.
void run_combined(int32_t gate, LweSample *res, const LweSample *a, const LweSample *b, const LweSample *c,
                  LweBootstrappingKeyFFT *f) {
    GateRequest req{gate, res, a, b, c, false};
    std::unique_lock<std::mutex> lk(f->comb_mu);
    f->comb_pending.push_back(&req);
    f->comb_arrive.notify_one();
    while (!req.done) {
        if (f->comb_busy) {
            f->comb_cv.wait(lk);
            continue;
        }
        f->comb_busy = true;
        if (f->comb_pending.size() < f->comb_last)
            f->comb_arrive.wait_for(lk, kGatherWait, [&] { return f->comb_pending.size() >= f->comb_last; });
        f->comb_last = f->comb_pending.size();
        std::vector<GateRequest *> batch;
        batch.swap(f->comb_pending);
        lk.unlock();
        evaluate_requests(f, batch);  // aborts on failure, like the reference's gates
        lk.lock();
        for (GateRequest *r : batch) r->done = true;
        f->comb_busy = false;
        f->comb_cv.notify_all();
    }
}

void pack(std::vector<int32_t> &buf, const LweSample *s, int32_t count, int32_t n) {
    buf.resize((size_t)count * (n + 1));
    for (int32_t g = 0; g < count; g++) {
        std::memcpy(&buf[(size_t)g * (n + 1)], s[g].a, sizeof(int32_t) * n);
        buf[(size_t)g * (n + 1) + n] = s[g].b;
    }
}

void unpack(LweSample *s, const std::vector<int32_t> &buf, int32_t count, int32_t n) {
    for (int32_t g = 0; g < count; g++) {
        std::memcpy(s[g].a, &buf[(size_t)g * (n + 1)], sizeof(int32_t) * n);
        s[g].b = buf[(size_t)g * (n + 1) + n];
        s[g].current_variance = 0.;
    }
}

void run_batch(int32_t gate, LweSample *res, const LweSample *a, const LweSample *b, const LweSample *c,
               int32_t count, const TFheGateBootstrappingCloudKeySet *bk) {
    const int32_t n = bk->params->in_out_params->n;
    if (gate == TFHEB_NOT || gate == TFHEB_COPY) {  // bootstrap-free (boot-gates.cpp:164-178)
        for (int32_t g = 0; g < count; g++) {
            for (int32_t i = 0; i < n; i++) res[g].a[i] = gate == TFHEB_NOT ? (int32_t)(0u - (uint32_t)a[g].a[i]) : a[g].a[i];
            res[g].b = gate == TFHEB_NOT ? (int32_t)(0u - (uint32_t)a[g].b) : a[g].b;
            res[g].current_variance = a[g].current_variance;
        }
        return;
    }
    LweBootstrappingKeyFFT *f = ready(bk);
    if (count == 1) {
        run_combined(gate, res, a, b, c, f);
        return;
    }
    std::vector<int32_t> ha, hb, hc, out((size_t)count * (n + 1));
    pack(ha, a, count, n);
    pack(hb, b, count, n);
    if (gate == TFHEB_MUX) pack(hc, c, count, n);
    if (tfheb_gate_batch(f->ck, gate, g_precision, count, ha.data(), hb.data(), gate == TFHEB_MUX ? hc.data() : nullptr,
                         out.data()) != TFHEB_OK)
        die("gate evaluation");
    unpack(res, out, count, n);  // inputs were copied first, so res may alias a, b or c
}

}  // namespace

extern "C" {

TFheGateBootstrappingParameterSet *new_default_gate_bootstrapping_parameters(int32_t minimum_lambda) {
    tfheb_params p;
    if (tfheb_default_params(minimum_lambda, &p) != TFHEB_OK)
        die("the requested security parameter must be in (0, 128]");
    return make_params(p, 0.012467, 0.012467);
}

void delete_gate_bootstrapping_parameters(TFheGateBootstrappingParameterSet *params) {
    if (!params) return;
    std::free(const_cast<Torus32 *>(params->tgsw_params->h));
    std::free(const_cast<TLweParams *>(params->tgsw_params->tlwe_params));
    std::free(const_cast<TGswParams *>(params->tgsw_params));
    std::free(const_cast<LweParams *>(params->in_out_params));
    std::free(params);
}

TFheGateBootstrappingSecretKeySet *new_random_gate_bootstrapping_secret_keyset(
    const TFheGateBootstrappingParameterSet *params) {
    const tfheb_params p = to_params(params);
    tfheb_secret_key *sk = nullptr;
    tfheb_cloud_key *ck = nullptr;
    if (tfheb_keygen(&p, next_seed(), &sk, &ck) != TFHEB_OK) die("key generation");
    return assemble_secret_keyset(params, sk, ck);
}

void delete_gate_bootstrapping_cloud_keyset(TFheGateBootstrappingCloudKeySet *keyset) {
    if (!keyset) return;
    auto *f = const_cast<LweBootstrappingKeyFFT *>(keyset->bkFFT);
    auto *b = const_cast<LweBootstrappingKey *>(keyset->bk);
    if (f) {
        tfheb_cloud_key_free(f->ck);
        delete f;
    }
    delete b;
    std::free(keyset);
}

void delete_gate_bootstrapping_secret_keyset(TFheGateBootstrappingSecretKeySet *keyset) {
    if (!keyset) return;
    auto *f = const_cast<LweBootstrappingKeyFFT *>(keyset->cloud.bkFFT);
    if (f) {
        tfheb_cloud_key_free(f->ck);
        delete f;
    }
    delete const_cast<LweBootstrappingKey *>(keyset->cloud.bk);
    auto *gk = const_cast<TGswKey *>(keyset->tgsw_key);
    if (gk) {
        tfheb_secret_key_free(gk->sk);
        delete gk;
    }
    if (keyset->lwe_key) {
        std::free(keyset->lwe_key->key);
        std::free(const_cast<LweKey *>(keyset->lwe_key));
    }
    std::free(keyset);
}

LweSample *new_gate_bootstrapping_ciphertext(const TFheGateBootstrappingParameterSet *params) {
    return new_gate_bootstrapping_ciphertext_array(1, params);
}

LweSample *new_gate_bootstrapping_ciphertext_array(int32_t nbelems, const TFheGateBootstrappingParameterSet *params) {
    const int32_t n = params->in_out_params->n;
    LweSample *s = static_cast<LweSample *>(std::malloc(sizeof(LweSample) * (size_t)nbelems));
    for (int32_t i = 0; i < nbelems; i++) {
        s[i].a = static_cast<Torus32 *>(std::calloc((size_t)n, sizeof(Torus32)));
        s[i].b = 0;
        s[i].current_variance = 0.;
    }
    return s;
}

void delete_gate_bootstrapping_ciphertext(LweSample *sample) { delete_gate_bootstrapping_ciphertext_array(1, sample); }

void delete_gate_bootstrapping_ciphertext_array(int32_t nbelems, LweSample *samples) {
    if (!samples) return;
    for (int32_t i = 0; i < nbelems; i++) std::free(samples[i].a);
    std::free(samples);
}

void bootsSymEncrypt(LweSample *result, int32_t message, const TFheGateBootstrappingSecretKeySet *key) {
    const int32_t n = key->params->in_out_params->n;
    std::vector<int32_t> ct(n + 1);
    const int32_t bit = message ? 1 : 0;
    if (tfheb_encrypt(key->tgsw_key->sk, &bit, 1, next_seed(), ct.data()) != TFHEB_OK) die("encryption");
    std::memcpy(result->a, ct.data(), sizeof(int32_t) * n);
    result->b = ct[n];
    const double alpha = key->params->in_out_params->alpha_min;
    result->current_variance = alpha * alpha;
}

int32_t bootsSymDecrypt(const LweSample *sample, const TFheGateBootstrappingSecretKeySet *key) {
    return lwePhase(sample, key->lwe_key) > 0 ? 1 : 0;
}

void bootsCONSTANT(LweSample *result, int32_t value, const TFheGateBootstrappingCloudKeySet *bk) {
    const int32_t n = bk->params->in_out_params->n;
    const Torus32 mu = modSwitchToTorus32(1, 8);
    std::memset(result->a, 0, sizeof(int32_t) * n);
    result->b = value ? mu : (Torus32)(0u - (uint32_t)mu);
    result->current_variance = 0.;
}

#define TFHE_B200_BINARY_GATE(NAME, CODE)                                                              \
    void NAME(LweSample *result, const LweSample *ca, const LweSample *cb, const TFheGateBootstrappingCloudKeySet *bk) { \
        run_batch(CODE, result, ca, cb, nullptr, 1, bk);                                               \
    }
TFHE_B200_BINARY_GATE(bootsNAND, TFHEB_NAND)
TFHE_B200_BINARY_GATE(bootsOR, TFHEB_OR)
TFHE_B200_BINARY_GATE(bootsAND, TFHEB_AND)
TFHE_B200_BINARY_GATE(bootsXOR, TFHEB_XOR)
TFHE_B200_BINARY_GATE(bootsXNOR, TFHEB_XNOR)
TFHE_B200_BINARY_GATE(bootsNOR, TFHEB_NOR)
TFHE_B200_BINARY_GATE(bootsANDNY, TFHEB_ANDNY)
TFHE_B200_BINARY_GATE(bootsANDYN, TFHEB_ANDYN)
TFHE_B200_BINARY_GATE(bootsORNY, TFHEB_ORNY)
TFHE_B200_BINARY_GATE(bootsORYN, TFHEB_ORYN)
#undef TFHE_B200_BINARY_GATE

void bootsNOT(LweSample *result, const LweSample *ca, const TFheGateBootstrappingCloudKeySet *bk) {
    run_batch(TFHEB_NOT, result, ca, nullptr, nullptr, 1, bk);
}

void bootsCOPY(LweSample *result, const LweSample *ca, const TFheGateBootstrappingCloudKeySet *bk) {
    run_batch(TFHEB_COPY, result, ca, nullptr, nullptr, 1, bk);
}

void bootsMUX(LweSample *result, const LweSample *a, const LweSample *b, const LweSample *c,
              const TFheGateBootstrappingCloudKeySet *bk) {
    run_batch(TFHEB_MUX, result, a, b, c, 1, bk);
}

void bootsGATE_batch(int32_t gate, LweSample *results, const LweSample *a, const LweSample *b, const LweSample *c,
                     int32_t count, const TFheGateBootstrappingCloudKeySet *bk) {
    if (gate < 0 || gate > TFHEB_COPY || count < 0) die("bootsGATE_batch: bad gate code or count");
    run_batch(gate, results, a, b, c, count, bk);
}

void bootsNAND_batch(LweSample *results, const LweSample *a, const LweSample *b, int32_t count,
                     const TFheGateBootstrappingCloudKeySet *bk) {
    run_batch(TFHEB_NAND, results, a, b, nullptr, count, bk);
}

void bootsMUX_batch(LweSample *results, const LweSample *a, const LweSample *b, const LweSample *c, int32_t count,
                    const TFheGateBootstrappingCloudKeySet *bk) {
    run_batch(TFHEB_MUX, results, a, b, c, count, bk);
}

void tfhe_random_generator_setSeed(uint32_t *values, int32_t size) {
    std::lock_guard<std::mutex> lock(g_rng_mu);
    uint64_t h = 0x84222325CBF29CE4ull;
    for (int32_t i = 0; i < size; i++) h = (h ^ values[i]) * 0x100000001B3ull;
    g_rng_state = h;
}

void tfhe_b200_set_precision(int32_t precision) {
    if (precision != TFHEB_FP64 && precision != TFHEB_SPLIT_FP32) die("tfhe_b200_set_precision: unknown precision");
    g_precision = precision;
}

Torus32 modSwitchToTorus32(int32_t mu, int32_t Msize) { return tfheb::modswitch_to_torus32(mu, Msize); }

int32_t modSwitchFromTorus32(Torus32 phase, int32_t Msize) { return tfheb::modswitch_from_torus32(phase, Msize); }

Torus32 lwePhase(const LweSample *sample, const LweKey *key) {
    uint32_t axs = 0;
    for (int32_t i = 0; i < key->params->n; i++) axs += (uint32_t)sample->a[i] * (uint32_t)key->key[i];
    return (Torus32)((uint32_t)sample->b - axs);
}

// Single-sample bootstraps through the batched device entry points (lwe-bootstrapping-functions-fft.cpp:169-225).
static void bootstrap_one(LweSample *result, const LweBootstrappingKeyFFT *bkc, Torus32 mu, const LweSample *x,
                          bool with_ks) {
    auto *f = const_cast<LweBootstrappingKeyFFT *>(bkc);
    ensure_on_device(f);
    const int32_t n = f->n, out_n = with_ks ? f->n : f->kN;
    std::vector<int32_t> in(n + 1), out(out_n + 1);
    std::memcpy(in.data(), x->a, sizeof(int32_t) * n);
    in[n] = x->b;
    int32_t *d_in = nullptr, *d_out = nullptr;
    if (cudaMalloc(&d_in, in.size() * 4) != cudaSuccess || cudaMalloc(&d_out, out.size() * 4) != cudaSuccess)
        die("device allocation");
    cudaMemcpy(d_in, in.data(), in.size() * 4, cudaMemcpyHostToDevice);
    const tfheb_status st = with_ks ? tfheb_bootstrap_device(f->ck, g_precision, mu, 1, d_in, d_out, nullptr)
                                    : tfheb_bootstrap_woks_device(f->ck, g_precision, mu, 1, d_in, d_out, nullptr);
    if (st != TFHEB_OK || tfheb_synchronize(f->ck) != TFHEB_OK) die("bootstrap");
    cudaMemcpy(out.data(), d_out, out.size() * 4, cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_out);
    std::memcpy(result->a, out.data(), sizeof(int32_t) * out_n);
    result->b = out[out_n];
    result->current_variance = 0.;
}

void tfhe_bootstrap_FFT(LweSample *result, const LweBootstrappingKeyFFT *bk, Torus32 mu, const LweSample *x) {
    bootstrap_one(result, bk, mu, x, true);
}

void tfhe_bootstrap_woKS_FFT(LweSample *result, const LweBootstrappingKeyFFT *bk, Torus32 mu, const LweSample *x) {
    bootstrap_one(result, bk, mu, x, false);
}

// The coefficient-domain entry points (lwe-bootstrapping-functions.cpp:138-179) run the same GPU
// path on the same key: the reference computes their external products exactly with integer
// polynomial products, this library through its FFT (FP64 by default), so a result may differ
// from the reference's by a few Torus32 units while decrypting the same.
static void bootstrap_coef(LweSample *result, const LweBootstrappingKey *bk, Torus32 mu, const LweSample *x,
                           bool with_ks) {
    if (!bk || !bk->ck) die("bootstrapping key is empty");
    tfheb_params p;
    tfheb_cloud_key_params(bk->ck, &p);
    const LweBootstrappingKeyFFT view(bk->ck, p.n, p.k * p.N);  // moves missing device keys once
    bootstrap_one(result, &view, mu, x, with_ks);
}

void tfhe_bootstrap(LweSample *result, const LweBootstrappingKey *bk, Torus32 mu, const LweSample *x) {
    bootstrap_coef(result, bk, mu, x, true);
}

void tfhe_bootstrap_woKS(LweSample *result, const LweBootstrappingKey *bk, Torus32 mu, const LweSample *x) {
    bootstrap_coef(result, bk, mu, x, false);
}

// ---- LWE helpers of lwe-functions.h (lwe-functions.cpp:33-178), host side -------------------

void lweSymEncrypt(LweSample *result, Torus32 message, double alpha, const LweKey *key) {
    const int32_t n = key->params->n;
    std::vector<int32_t> ct(n + 1);
    tfheb::encrypt_torus(n, key->key, &message, 1, alpha, next_seed(), ct.data());
    std::memcpy(result->a, ct.data(), sizeof(int32_t) * n);
    result->b = ct[n];
    result->current_variance = alpha * alpha;
}

void lweSymEncryptWithExternalNoise(LweSample *result, Torus32 message, double noise, double alpha,
                                    const LweKey *key) {
    const int32_t n = key->params->n;
    const Torus32 mu = (Torus32)((uint32_t)message + (uint32_t)tfheb::double_to_torus32(noise));
    std::vector<int32_t> ct(n + 1);
    tfheb::encrypt_torus(n, key->key, &mu, 1, 0.0, next_seed(), ct.data());
    std::memcpy(result->a, ct.data(), sizeof(int32_t) * n);
    result->b = ct[n];
    result->current_variance = alpha * alpha;
}

Torus32 approxPhase(Torus32 phase, int32_t Msize) { return tfheb::approx_phase(phase, Msize); }

Torus32 lweSymDecrypt(const LweSample *sample, const LweKey *key, const int32_t Msize) {
    return tfheb::approx_phase(lwePhase(sample, key), Msize);
}

void lweClear(LweSample *result, const LweParams *params) {
    std::memset(result->a, 0, sizeof(int32_t) * params->n);
    result->b = 0;
    result->current_variance = 0.;
}

void lweCopy(LweSample *result, const LweSample *sample, const LweParams *params) {
    std::memmove(result->a, sample->a, sizeof(int32_t) * params->n);
    result->b = sample->b;
    result->current_variance = sample->current_variance;
}

void lweNegate(LweSample *result, const LweSample *sample, const LweParams *params) {
    for (int32_t i = 0; i < params->n; i++) result->a[i] = (int32_t)(0u - (uint32_t)sample->a[i]);
    result->b = (int32_t)(0u - (uint32_t)sample->b);
    result->current_variance = sample->current_variance;
}

void lweNoiselessTrivial(LweSample *result, Torus32 mu, const LweParams *params) {
    std::memset(result->a, 0, sizeof(int32_t) * params->n);
    result->b = mu;
    result->current_variance = 0.;
}

// result += p * sample (p = 1, -1 for lweAddTo / lweSubTo), variance += p^2 * variance
static void lwe_add_mul(LweSample *result, int32_t p, const LweSample *sample, const LweParams *params) {
    for (int32_t i = 0; i < params->n; i++)
        result->a[i] = (int32_t)((uint32_t)result->a[i] + (uint32_t)p * (uint32_t)sample->a[i]);
    result->b = (int32_t)((uint32_t)result->b + (uint32_t)p * (uint32_t)sample->b);
    result->current_variance += (double)p * (double)p * sample->current_variance;
}

void lweAddTo(LweSample *result, const LweSample *sample, const LweParams *params) {
    lwe_add_mul(result, 1, sample, params);
}
void lweSubTo(LweSample *result, const LweSample *sample, const LweParams *params) {
    lwe_add_mul(result, -1, sample, params);
}
void lweAddMulTo(LweSample *result, int32_t p, const LweSample *sample, const LweParams *params) {
    lwe_add_mul(result, p, sample, params);
}
void lweSubMulTo(LweSample *result, int32_t p, const LweSample *sample, const LweParams *params) {
    lwe_add_mul(result, -p, sample, params);
}

}  // extern "C"

// ================================================================================================
// files in the reference's format (tfhe_io.cpp:90-136, 1010-1220)
// ================================================================================================

namespace {

// Parameter sets read together with a key set belong to the library, as the reference registers
// them with its garbage collector (tfhe_io.cpp:1103-1110, 1157-1164); they are freed at exit.
struct OwnedParams {
    std::mutex mu;
    std::vector<TFheGateBootstrappingParameterSet *> sets;
    ~OwnedParams() {
        for (auto *p : sets) delete_gate_bootstrapping_parameters(p);
    }
} g_owned_params;

tfheb::ParamMeta meta_of(const TFheGateBootstrappingParameterSet *ps) {
    return {ps->in_out_params->alpha_max, ps->tgsw_params->tlwe_params->alpha_max};
}

TFheGateBootstrappingParameterSet *read_params_or_die(FILE *F, tfheb::ParamMeta &m) {
    tfheb_params p{};
    if (!F || !tfheb::io::read_params(F, p, m)) die("reading a gate-bootstrapping parameter set");
    return make_params(p, m.in_alpha_max, m.tlwe_alpha_max);
}

const TFheGateBootstrappingParameterSet *read_owned_params(FILE *F, tfheb::ParamMeta &m) {
    TFheGateBootstrappingParameterSet *ps = read_params_or_die(F, m);
    std::lock_guard<std::mutex> lock(g_owned_params.mu);
    g_owned_params.sets.push_back(ps);
    return ps;
}

tfheb_cloud_key *read_cloud_or_die(FILE *F, const TFheGateBootstrappingParameterSet *ps, const tfheb::ParamMeta &m) {
    auto *c = new tfheb_cloud_key();
    c->ck.meta = m;
    tfheb_params p = to_params(ps);
    if (!tfheb::io::read_cloud_content(F, p, c->ck)) die("reading a bootstrapping key");
    return c;
}

void write_params_or_die(FILE *F, const TFheGateBootstrappingParameterSet *ps) {
    if (!F || !tfheb::io::write_params(F, to_params(ps), meta_of(ps))) die("writing a parameter set");
}

void write_cloud_or_die(FILE *F, const TFheGateBootstrappingCloudKeySet *ks) {
    if (!ks->bkFFT || !ks->bkFFT->ck) die("cloud keyset has no key");
    if (!tfheb::io::write_cloud_content(F, ks->bkFFT->ck->ck)) die("writing a bootstrapping key");
}

}  // namespace

extern "C" {

void export_lweSample_toFile(FILE *F, const LweSample *sample, const LweParams *params) {
    if (!F || !tfheb::io::write_lwe_sample(F, params->n, sample->a, sample->b, sample->current_variance))
        die("writing a LWE sample");
}

void import_lweSample_fromFile(FILE *F, LweSample *sample, const LweParams *params) {
    if (!F || !tfheb::io::read_lwe_sample(F, params->n, sample->a, &sample->b, &sample->current_variance))
        die("reading a LWE sample");
}

void export_gate_bootstrapping_ciphertext_toFile(FILE *F, const LweSample *sample,
                                                 const TFheGateBootstrappingParameterSet *params) {
    export_lweSample_toFile(F, sample, params->in_out_params);
}

void import_gate_bootstrapping_ciphertext_fromFile(FILE *F, LweSample *sample,
                                                   const TFheGateBootstrappingParameterSet *params) {
    import_lweSample_fromFile(F, sample, params->in_out_params);
}

void export_tfheGateBootstrappingParameterSet_toFile(FILE *F, const TFheGateBootstrappingParameterSet *params) {
    write_params_or_die(F, params);
}

TFheGateBootstrappingParameterSet *new_tfheGateBootstrappingParameterSet_fromFile(FILE *F) {
    tfheb::ParamMeta m;
    return read_params_or_die(F, m);
}

void export_tfheGateBootstrappingCloudKeySet_toFile(FILE *F, const TFheGateBootstrappingCloudKeySet *keyset) {
    write_params_or_die(F, keyset->params);
    write_cloud_or_die(F, keyset);
}

TFheGateBootstrappingCloudKeySet *new_tfheGateBootstrappingCloudKeySet_fromFile(FILE *F) {
    tfheb::ParamMeta m;
    const TFheGateBootstrappingParameterSet *ps = read_owned_params(F, m);
    return make(assemble_cloud(ps, read_cloud_or_die(F, ps, m)));
}

void export_tfheGateBootstrappingSecretKeySet_toFile(FILE *F, const TFheGateBootstrappingSecretKeySet *keyset) {
    write_params_or_die(F, keyset->params);
    write_cloud_or_die(F, &keyset->cloud);
    if (!keyset->tgsw_key || !tfheb::io::write_secret_content(F, keyset->tgsw_key->sk->sk))
        die("writing the secret keys");
}

TFheGateBootstrappingSecretKeySet *new_tfheGateBootstrappingSecretKeySet_fromFile(FILE *F) {
    tfheb::ParamMeta m;
    const TFheGateBootstrappingParameterSet *ps = read_owned_params(F, m);
    tfheb_cloud_key *ck = read_cloud_or_die(F, ps, m);
    auto *sk = new tfheb_secret_key();
    if (!tfheb::io::read_secret_content(F, ck->ck.p, sk->sk)) die("reading the secret keys");
    return assemble_secret_keyset(ps, sk, ck);
}

}  // extern "C"
