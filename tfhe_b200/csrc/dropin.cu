// dropin.cu -- the reference's gate-bootstrapping C API (include/tfhe.h) on top of the engine.
//
// Same symbols and caller-visible struct layouts as tfhe v1.1 (tfhe_gate_bootstrapping_functions.h,
// tfhe_gate_bootstrapping_structures.h, tfhe.h, lwebootstrappingkey.h); errors keep the reference's
// convention of void functions that abort on a fatal condition (tfhe_gate_bootstrapping.cpp:11-15
// die_dramatically).
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <mutex>
#include <type_traits>
#include <vector>

#include "../../include/tfhe.h"
#include "internal.h"

struct TGswKey {
    tfheb_secret_key *sk;
};

struct DropinKeys;

// A keyswitching key handle: the engine key it belongs to.
struct LweKeySwitchKey {
    DropinKeys *owner;
};
// One FFT-domain TGSW row of a key; the row itself lives on the GPU.
struct TLweSampleFFT {
    DropinKeys *owner;
    int32_t step, row;
};

namespace {

// One single-gate call waiting to be evaluated (see run_combined).
struct GateRequest {
    int32_t gate;
    LweSample *res;
    const LweSample *a, *b, *c;
    bool done;
};

// Pinned host and device buffers for single-sample calls; one call holds the lock from its upload
// to its synchronised download, so buffers grow (allocate) only when a larger call comes.
struct StagingArea {
    std::mutex mu;
    int32_t *h = nullptr, *d = nullptr;
    size_t cap = 0;
    ~StagingArea() {
        if (h) cudaFreeHost(h);
        if (d) cudaFree(d);
    }
};

}  // namespace

// Everything the drop-in keeps per cloud keyset: the engine key, the state of combined single-gate
// calls, staging buffers, variance tables and the views behind the public key structs.
struct DropinKeys {
    tfheb_cloud_key *ck = nullptr;
    tfheb_params p{};
    int32_t kpl = 0;
    std::atomic<int32_t> on_device_mask{0};  // precisions whose FFT-domain key is on the device
    // single-gate calls from concurrent threads, combined into batches
    std::mutex comb_mu;
    std::condition_variable comb_cv;      // callers waiting for their results or their turn
    std::condition_variable comb_arrive;  // the batch's leader gathering requests
    std::vector<GateRequest *> comb_pending;
    bool comb_busy = false;
    size_t comb_last = 0;  // requests in the previous batch
    StagingArea stage;
    // ks_var_sum[t] = the keyswitching-key sample variance added t times in sequence, the way
    // lweKeySwitchTranslate_fromArray accumulates it (lwe-keyswitch-functions.cpp:123-127)
    std::vector<double> ks_var_sum;
    double bk_var = 0;  // variance of every bootstrapping-key row
    // public views
    LweKeySwitchKey ks{};
    TGswSampleFFT *fft_samples = nullptr;  // [n]
    TLweSampleFFT *fft_rows = nullptr;     // [n][kpl]
    TLweSampleFFT **fft_blocs = nullptr;   // [n][k+1]
    TGswSample *coef_samples = nullptr;    // [n]
    TLweSample *coef_rows = nullptr;       // [n][kpl]
    TLweSample **coef_blocs = nullptr;     // [n][k+1]
    TorusPolynomial *coef_polys = nullptr; // [n][kpl][k+1], into the key's host coefficients
};

namespace {

// The public key structs with the drop-in's state behind them; standard layout, public part first,
// so a pointer to the public struct converts back.
struct CoefKeyImpl {
    LweBootstrappingKey pub;
    DropinKeys *keys;
};
struct FftKeyImpl {
    LweBootstrappingKeyFFT pub;
    DropinKeys *keys;
};
static_assert(std::is_standard_layout<CoefKeyImpl>::value && std::is_standard_layout<FftKeyImpl>::value,
              "key wrappers must convert to and from their public part");

[[noreturn]] void die(const char *what) {
    std::fprintf(stderr, "tfhe_b200: %s: %s\n", what, tfheb_last_error());
    std::abort();
}

std::mutex g_rng_mu;
uint64_t g_rng_state = 0x243F6A8885A308D3ull;  // reseeded by tfhe_random_generator_setSeed
std::atomic<int32_t> g_precision{TFHEB_FP64};  // set by tfhe_b200_set_precision, read by every gate

// every live DropinKeys, to recognise a keyset's own coefficient-domain TGSW samples
std::mutex g_keys_mu;
std::vector<DropinKeys *> g_keys;

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
template <typename T>
void put_bytes(T *dst, const T &v) {  // assign an object with const members
    std::memcpy(static_cast<void *>(dst), &v, sizeof(T));
}
template <typename T>
T *alloc_array(size_t n) {
    T *p = static_cast<T *>(std::calloc(n ? n : 1, sizeof(T)));
    if (!p) die("host allocation");
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

// The drop-in state and public views of an engine key (the keyset owns ck).
DropinKeys *make_keys(const TFheGateBootstrappingParameterSet *params, tfheb_cloud_key *ck) {
    auto *k = new DropinKeys();
    k->ck = ck;
    k->p = to_params(params);
    const tfheb_params &p = k->p;
    const int32_t K = p.k, L = p.l, N = p.N, n = p.n, kpl = (K + 1) * L;
    k->kpl = kpl;
    const tfheb::CloudKey &c = ck->ck;
    // variances the reference gives its key samples: alpha^2 at key generation, the file's value
    // when read from a file (tfhe_io.cpp:796-812, 905-928)
    const double ks_var = c.ks_var >= 0 ? c.ks_var : p.ks_stdev * p.ks_stdev;
    k->bk_var = c.bk_var >= 0 ? c.bk_var : p.bk_stdev * p.bk_stdev;
    k->ks_var_sum.assign((size_t)K * N * p.ks_t + 1, 0.0);
    for (size_t t = 1; t < k->ks_var_sum.size(); t++) k->ks_var_sum[t] = k->ks_var_sum[t - 1] + ks_var;
    k->ks.owner = k;
    // FFT-domain views: handles (step, row)
    k->fft_samples = alloc_array<TGswSampleFFT>(n);
    k->fft_rows = alloc_array<TLweSampleFFT>((size_t)n * kpl);
    k->fft_blocs = alloc_array<TLweSampleFFT *>((size_t)n * (K + 1));
    for (int32_t i = 0; i < n; i++) {
        for (int32_t r = 0; r < kpl; r++) k->fft_rows[(size_t)i * kpl + r] = TLweSampleFFT{k, i, r};
        for (int32_t u = 0; u <= K; u++) k->fft_blocs[(size_t)i * (K + 1) + u] = &k->fft_rows[(size_t)i * kpl + u * L];
        put_bytes(&k->fft_samples[i],
                  TGswSampleFFT{&k->fft_rows[(size_t)i * kpl], &k->fft_blocs[(size_t)i * (K + 1)], K, L});
    }
    // coefficient-domain views into the key's host coefficients [n][kpl][k+1][N]
    if (!c.bsk_coef.empty()) {
        Torus32 *coef = const_cast<Torus32 *>(c.bsk_coef.data());
        k->coef_samples = alloc_array<TGswSample>(n);
        k->coef_rows = alloc_array<TLweSample>((size_t)n * kpl);
        k->coef_blocs = alloc_array<TLweSample *>((size_t)n * (K + 1));
        k->coef_polys = alloc_array<TorusPolynomial>((size_t)n * kpl * (K + 1));
        for (size_t r = 0; r < (size_t)n * kpl; r++) {
            for (int32_t u = 0; u <= K; u++)
                put_bytes(&k->coef_polys[r * (K + 1) + u], TorusPolynomial{N, coef + (r * (K + 1) + u) * N});
            TorusPolynomial *a = &k->coef_polys[r * (K + 1)];
            put_bytes(&k->coef_rows[r], TLweSample{a, a + K, k->bk_var, K});
        }
        for (int32_t i = 0; i < n; i++) {
            for (int32_t u = 0; u <= K; u++)
                k->coef_blocs[(size_t)i * (K + 1) + u] = &k->coef_rows[(size_t)i * kpl + u * L];
            put_bytes(&k->coef_samples[i],
                      TGswSample{&k->coef_rows[(size_t)i * kpl], &k->coef_blocs[(size_t)i * (K + 1)], K, L});
        }
    }
    std::lock_guard<std::mutex> lock(g_keys_mu);
    g_keys.push_back(k);
    return k;
}

void free_keys(DropinKeys *k) {
    if (!k) return;
    {
        std::lock_guard<std::mutex> lock(g_keys_mu);
        for (size_t i = 0; i < g_keys.size(); i++)
            if (g_keys[i] == k) {
                g_keys.erase(g_keys.begin() + i);
                break;
            }
    }
    std::free(k->fft_samples);
    std::free(k->fft_rows);
    std::free(k->fft_blocs);
    std::free(k->coef_samples);
    std::free(k->coef_rows);
    std::free(k->coef_blocs);
    std::free(k->coef_polys);
    tfheb_cloud_key_free(k->ck);
    delete k;
}

// The drop-in objects around an engine key pair (the keysets own sk and ck).
TFheGateBootstrappingCloudKeySet assemble_cloud(const TFheGateBootstrappingParameterSet *params, tfheb_cloud_key *ck) {
    DropinKeys *k = make_keys(params, ck);
    const TGswParams *gp = params->tgsw_params;
    const TLweParams *tp = gp->tlwe_params;
    auto *coef = make(CoefKeyImpl{LweBootstrappingKey{params->in_out_params, gp, tp, &tp->extracted_lweparams,
                                                      k->coef_samples, &k->ks},
                                  k});
    auto *fft = make(FftKeyImpl{LweBootstrappingKeyFFT{params->in_out_params, gp, tp, &tp->extracted_lweparams,
                                                       k->fft_samples, &k->ks},
                                k});
    return TFheGateBootstrappingCloudKeySet{params, &coef->pub, &fft->pub};
}
TFheGateBootstrappingSecretKeySet *assemble_secret_keyset(const TFheGateBootstrappingParameterSet *params,
                                                          tfheb_secret_key *sk, tfheb_cloud_key *ck) {
    const int32_t n = params->in_out_params->n;
    int32_t *key = static_cast<int32_t *>(std::malloc(sizeof(int32_t) * n));
    tfheb_secret_key_export(sk, key, nullptr);
    LweKey *lk = make(LweKey{params->in_out_params, key});
    return make(TFheGateBootstrappingSecretKeySet{params, lk, new TGswKey{sk}, assemble_cloud(params, ck)});
}

DropinKeys *keys_of(const LweBootstrappingKeyFFT *bk) {
    if (!bk) die("bootstrapping key is empty");
    return reinterpret_cast<const FftKeyImpl *>(bk)->keys;
}
DropinKeys *keys_of(const LweBootstrappingKey *bk) {
    if (!bk) die("bootstrapping key is empty");
    return reinterpret_cast<const CoefKeyImpl *>(bk)->keys;
}

// Frees the drop-in objects of a cloud keyset (not the keyset struct itself).
void free_cloud_parts(const TFheGateBootstrappingCloudKeySet *cs) {
    DropinKeys *k = cs->bkFFT ? keys_of(cs->bkFFT) : nullptr;
    std::free(const_cast<LweBootstrappingKeyFFT *>(cs->bkFFT));
    std::free(const_cast<LweBootstrappingKey *>(cs->bk));
    free_keys(k);
}

// Moves the key of the current precision to the device on first use.  Threads may race here on a
// fresh keyset: the transfer runs under the key's own lock and skips a precision already present,
// so a second caller only waits; the mask is atomic.
void ensure_on_device(DropinKeys *k) {
    const int32_t bit = 1 << g_precision;
    if (k->on_device_mask.load(std::memory_order_acquire) & bit) return;
    if (tfheb_cloud_key_to_device(k->ck, device_index(), bit, 0) != TFHEB_OK) die("moving the key to the GPU");
    k->on_device_mask.fetch_or(bit, std::memory_order_release);
}

DropinKeys *ready(const TFheGateBootstrappingCloudKeySet *bk) {
    if (!bk || !bk->bkFFT) die("cloud keyset has no key");
    DropinKeys *k = keys_of(bk->bkFFT);
    if (!k || !k->ck) die("cloud keyset has no key");
    ensure_on_device(k);
    return k;
}

// current_variance of a keyswitched result with `terms` non-zero digits
double ks_variance(const DropinKeys *k, int32_t terms) {
    if (terms < 0 || (size_t)terms >= k->ks_var_sum.size()) die("keyswitch term count out of range");
    return k->ks_var_sum[(size_t)terms];
}

// Evaluates a set of single-gate requests: one batch per gate code present.  Every request's
// operands are copied before its group's results are written, so a result may alias its own operands.
void evaluate_requests(DropinKeys *k, const std::vector<GateRequest *> &reqs) {
    const int32_t n = k->p.n, row = n + 1;
    for (int32_t code = 0; code < TFHEB_NOT; code++) {
        std::vector<GateRequest *> grp;
        for (GateRequest *r : reqs)
            if (r->gate == code) grp.push_back(r);
        if (grp.empty()) continue;
        const size_t cnt = grp.size();
        std::vector<int32_t> ha(cnt * row), hb(cnt * row), hc(code == TFHEB_MUX ? cnt * row : 0), out(cnt * row),
            terms(cnt);
        auto put = [&](std::vector<int32_t> &buf, size_t i, const LweSample *x) {
            std::memcpy(&buf[i * row], x->a, sizeof(int32_t) * n);
            buf[i * row + n] = x->b;
        };
        for (size_t i = 0; i < cnt; i++) {
            put(ha, i, grp[i]->a);
            put(hb, i, grp[i]->b);
            if (code == TFHEB_MUX) put(hc, i, grp[i]->c);
        }
        if (tfheb_gate_batch_terms(k->ck, code, g_precision, (int32_t)cnt, ha.data(), hb.data(),
                                   code == TFHEB_MUX ? hc.data() : nullptr, out.data(), terms.data()) != TFHEB_OK)
            die("gate evaluation");
        for (size_t i = 0; i < cnt; i++) {
            std::memcpy(grp[i]->res->a, &out[i * row], sizeof(int32_t) * n);
            grp[i]->res->b = out[i * row + n];
            grp[i]->res->current_variance = ks_variance(k, terms[i]);
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
                  DropinKeys *f) {
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
    DropinKeys *k = ready(bk);
    if (count == 1) {
        run_combined(gate, res, a, b, c, k);
        return;
    }
    std::vector<int32_t> ha, hb, hc, out((size_t)count * (n + 1)), terms(count);
    pack(ha, a, count, n);
    pack(hb, b, count, n);
    if (gate == TFHEB_MUX) pack(hc, c, count, n);
    if (tfheb_gate_batch_terms(k->ck, gate, g_precision, count, ha.data(), hb.data(),
                               gate == TFHEB_MUX ? hc.data() : nullptr, out.data(), terms.data()) != TFHEB_OK)
        die("gate evaluation");
    // inputs were copied first, so res may alias a, b or c
    for (int32_t g = 0; g < count; g++) {
        std::memcpy(res[g].a, &out[(size_t)g * (n + 1)], sizeof(int32_t) * n);
        res[g].b = out[(size_t)g * (n + 1) + n];
        res[g].current_variance = ks_variance(k, terms[g]);
    }
}

// ---- single-sample calls through staging buffers -------------------------------------------------

// Holds a staging area for one call: host and device words [0, words), copies on the key's stream,
// and a final synchronisation that reports device errors.  Growing the area allocates; a call of a
// size seen before allocates nothing.
class Staged {
  public:
    Staged(StagingArea &area, tfheb_cloud_key *ck, size_t words) : a_(area), lock_(area.mu), ck_(ck) {
        // the copies below run on the key's stream from whatever host thread calls: make its device
        // current here, not only when the buffers grow
        if (cudaSetDevice(ck->ck.device) != cudaSuccess) die("selecting the key's GPU");
        if (words > a_.cap) {
            if (a_.h) cudaFreeHost(a_.h);
            if (a_.d) cudaFree(a_.d);
            a_.h = a_.d = nullptr;
            a_.cap = 0;
            if (cudaMallocHost((void **)&a_.h, words * 4) != cudaSuccess || cudaMalloc((void **)&a_.d, words * 4) != cudaSuccess)
                die("staging buffers");
            a_.cap = words;
        }
    }
    int32_t *h(size_t off) { return a_.h + off; }
    int32_t *d(size_t off) { return a_.d + off; }
    void up(size_t off, size_t words) {
        if (cudaMemcpyAsync(d(off), h(off), words * 4, cudaMemcpyHostToDevice, ck_->ck.stream) != cudaSuccess)
            die("copy to the GPU");
    }
    void down(size_t off, size_t words) {
        if (cudaMemcpyAsync(h(off), d(off), words * 4, cudaMemcpyDeviceToHost, ck_->ck.stream) != cudaSuccess)
            die("copy from the GPU");
    }
    void finish(const char *what) {
        if (tfheb::sync_key_stream(ck_) != TFHEB_OK) die(what);
    }

  private:
    StagingArea &a_;
    std::lock_guard<std::mutex> lock_;
    tfheb_cloud_key *ck_;
};

void load_lwe(int32_t *dst, const LweSample *x, int32_t n) {
    std::memcpy(dst, x->a, sizeof(int32_t) * n);
    dst[n] = x->b;
}
void store_lwe(LweSample *r, const int32_t *src, int32_t n) {
    std::memcpy(r->a, src, sizeof(int32_t) * n);
    r->b = src[n];
}
void load_tlwe(int32_t *dst, const TLweSample *x, int32_t k, int32_t N) {
    for (int32_t u = 0; u <= k; u++) std::memcpy(dst + (size_t)u * N, x->a[u].coefsT, sizeof(int32_t) * N);
}
void store_tlwe(TLweSample *r, const int32_t *src, int32_t k, int32_t N) {
    for (int32_t u = 0; u <= k; u++) std::memcpy(r->a[u].coefsT, src + (size_t)u * N, sizeof(int32_t) * N);
}

// Single-sample bootstrap (lwe-bootstrapping-functions-fft.cpp:169-225): the extracted sample, and
// with_ks its keyswitch.  The keyswitched result's variance is the reference's digit-count sum; the
// extraction leaves the variance of `result` as it was (lwe.cpp:41-53 does not set it).
void bootstrap_one(LweSample *result, DropinKeys *k, Torus32 mu, const LweSample *x, bool with_ks) {
    ensure_on_device(k);
    const int32_t n = k->p.n, kN = k->p.k * k->p.N;
    const size_t o_in = 0, o_u = o_in + n + 1, o_out = o_u + kN + 1, o_terms = o_out + n + 1;
    Staged st(k->stage, k->ck, o_terms + 1);
    load_lwe(st.h(o_in), x, n);
    st.up(o_in, n + 1);
    if (tfheb_bootstrap_woks_device(k->ck, g_precision, mu, 1, st.d(o_in), st.d(o_u), nullptr) != TFHEB_OK)
        die("bootstrap");
    if (with_ks) {
        if (tfheb_keyswitch_device(k->ck, 1, st.d(o_u), st.d(o_out), nullptr) != TFHEB_OK ||
            tfheb_ks_terms_device(k->ck, 1, st.d(o_u), st.d(o_terms), nullptr) != TFHEB_OK)
            die("keyswitch");
        st.down(o_out, n + 2);  // the output and its term count
    } else {
        st.down(o_u, kN + 1);
    }
    st.finish("bootstrap");
    if (with_ks) {
        store_lwe(result, st.h(o_out), n);
        result->current_variance = ks_variance(k, *st.h(o_terms));
    } else {
        store_lwe(result, st.h(o_u), kN);
    }
}

// The owner and first step of TGSW samples that belong to a keyset's coefficient-domain view.
bool own_coef_samples(const TGswSample *bk, int32_t n, DropinKeys **owner, int32_t *first) {
    if (!bk) return false;
    std::lock_guard<std::mutex> lock(g_keys_mu);
    for (DropinKeys *k : g_keys) {
        if (!k->coef_samples) continue;
        if (bk >= k->coef_samples && bk < k->coef_samples + k->p.n) {
            *owner = k;
            *first = (int32_t)(bk - k->coef_samples);
            if (*first + n > k->p.n) die("blind rotation past the last TGSW sample of the key");
            return true;
        }
    }
    return false;
}

// The owner and first step of FFT-domain TGSW samples (they always come from a keyset).
DropinKeys *own_fft_samples(const TGswSampleFFT *bk, int32_t n, int32_t *first) {
    if (!bk || !bk->all_samples || !bk->all_samples->owner) die("FFT-domain TGSW samples without a key");
    DropinKeys *k = bk->all_samples->owner;
    *first = bk->all_samples->step;
    if (*first < 0 || *first + n > k->p.n) die("blind rotation past the last TGSW sample of the key");
    return k;
}

// An engine key holding caller-made coefficient-domain TGSW samples bk[0..n-1] (no keyswitching
// key), on the device in the current precision.  The caller frees it.
tfheb_cloud_key *temporary_key(const TGswSample *bk, int32_t n, const TGswParams *gp) {
    const TLweParams *tp = gp->tlwe_params;
    const int32_t K = tp->k, N = tp->N, L = gp->l, kpl = (K + 1) * L;
    // a rotation over no TGSW sample still needs a key of the right shape: one zero sample
    tfheb_params p{n > 0 ? n : 1, N, K, L, gp->Bgbit, 8, 2, tp->alpha_min, tp->alpha_min};
    std::vector<int32_t> coef((size_t)p.n * kpl * (K + 1) * N, 0);
    for (int32_t i = 0; i < n; i++)
        for (int32_t r = 0; r < kpl; r++)
            for (int32_t u = 0; u <= K; u++)
                std::memcpy(&coef[(((size_t)i * kpl + r) * (K + 1) + u) * N], bk[i].all_sample[r].a[u].coefsT,
                            sizeof(int32_t) * N);
    tfheb_cloud_key *ck = nullptr;
    if (tfheb_cloud_key_import(&p, coef.data(), nullptr, &ck) != TFHEB_OK) die("TGSW samples");
    if (tfheb_cloud_key_to_device(ck, device_index(), 1 << g_precision, 0) != TFHEB_OK) die("moving TGSW samples to the GPU");
    return ck;
}

// tfhe_blindRotate(_FFT) body: accum rotated by the TGSW samples first .. first+n-1 of an engine key
// (its staging area, or a temporary one for a temporary key).  The variance stays accum's: the
// reference's steps replace it by the previous accumulator's (lwe-bootstrapping-functions-fft.cpp:
// 67-76, tlwe-fft-operations.cpp:65-85).
void blind_rotate_on(tfheb_cloud_key *ck, StagingArea &area, int32_t first, TLweSample *accum, const int32_t *bara,
                     int32_t n, int32_t K, int32_t N) {
    if (n == 0) return;
    const size_t tl = (size_t)(K + 1) * N;
    Staged st(area, ck, tl + n);
    load_tlwe(st.h(0), accum, K, N);
    std::memcpy(st.h(tl), bara, sizeof(int32_t) * n);
    st.up(0, tl + n);
    if (tfheb_blind_rotate_steps_device(ck, g_precision, 1, first, n, st.d(tl), st.d(0), nullptr) != TFHEB_OK)
        die("blind rotation");
    st.down(0, tl);
    st.finish("blind rotation");
    store_tlwe(accum, st.h(0), K, N);
}

// tfhe_blindRotateAndExtract(_FFT) body; result's variance is left as it was (lwe.cpp:41-53).
void rotate_extract_on(tfheb_cloud_key *ck, StagingArea &area, int32_t first, LweSample *result,
                       const TorusPolynomial *v, int32_t barb, const int32_t *bara, int32_t n, int32_t K, int32_t N) {
    const size_t o_v = 0, o_barb = N, o_bara = o_barb + 1, o_out = o_bara + n;
    Staged st(area, ck, o_out + (size_t)K * N + 1);
    std::memcpy(st.h(o_v), v->coefsT, sizeof(int32_t) * N);
    *st.h(o_barb) = barb;
    if (n) std::memcpy(st.h(o_bara), bara, sizeof(int32_t) * n);
    st.up(0, o_out);
    if (tfheb_blind_rotate_extract_device(ck, g_precision, 1, first, n, st.d(o_v), st.d(o_barb), st.d(o_bara),
                                          st.d(o_out), nullptr) != TFHEB_OK)
        die("blind rotation and extraction");
    st.down(o_out, (size_t)K * N + 1);
    st.finish("blind rotation and extraction");
    store_lwe(result, st.h(o_out), K * N);
}

// ||digits||^2 of the gadget decomposition of one polynomial (tgsw-functions.cpp:297-410 digits,
// intPolynomialNormSq2 of toruspolynomial-functions.cpp:174-183): the reference's variance bookkeeping.
double digit_norm_sq(const Torus32 *poly, int32_t N, const TGswParams *gp, int32_t q) {
    const uint32_t shift = 32 - (q + 1) * gp->Bgbit;
    int32_t s = 0;
    for (int32_t j = 0; j < N; j++) {
        const int32_t d = (int32_t)((((uint32_t)poly[j] + gp->offset) >> shift) & gp->maskMod) - gp->halfBg;
        s += d * d;
    }
    return s;
}

// result = a (x) b on the GPU; the variance as tGswExternProduct / tGswExternMulToTLwe keep it:
// sum over rows of ||digit row||^2 * row variance (tlwe-functions.cpp:191-197), plus b's when add_b.
void extern_product(TLweSample *result, const TGswSample *a, const TLweSample *b, const TGswParams *gp, bool add_b) {
    const TLweParams *tp = gp->tlwe_params;
    const int32_t K = tp->k, N = tp->N, L = gp->l;
    double var = 0;
    for (int32_t u = 0; u <= K; u++)
        for (int32_t q = 0; q < L; q++)
            var += digit_norm_sq(b->a[u].coefsT, N, gp, q) * a->all_sample[u * L + q].current_variance;
    if (add_b) var += b->current_variance;
    auto run = [&](tfheb_cloud_key *ck, StagingArea &area, int32_t step) {
        const size_t tl = (size_t)(K + 1) * N;
        Staged st(area, ck, 2 * tl);
        load_tlwe(st.h(0), b, K, N);
        st.up(0, tl);
        if (tfheb_extern_product_device(ck, g_precision, 1, step, st.d(0), st.d(tl), nullptr) != TFHEB_OK)
            die("external product");
        st.down(tl, tl);
        st.finish("external product");
        store_tlwe(result, st.h(tl), K, N);
    };
    DropinKeys *owner = nullptr;
    int32_t step = 0;
    if (own_coef_samples(a, 1, &owner, &step)) {
        ensure_on_device(owner);
        run(owner->ck, owner->stage, step);
    } else {
        tfheb_cloud_key *ck = temporary_key(a, 1, gp);
        {
            StagingArea area;
            run(ck, area, 0);
        }
        tfheb_cloud_key_free(ck);
    }
    result->current_variance = var;
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
    free_cloud_parts(keyset);
    std::free(keyset);
}

void delete_gate_bootstrapping_secret_keyset(TFheGateBootstrappingSecretKeySet *keyset) {
    if (!keyset) return;
    free_cloud_parts(&keyset->cloud);
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
    return new_LweSample_array(nbelems, params->in_out_params);
}

void delete_gate_bootstrapping_ciphertext(LweSample *sample) { delete_gate_bootstrapping_ciphertext_array(1, sample); }

void delete_gate_bootstrapping_ciphertext_array(int32_t nbelems, LweSample *samples) {
    delete_LweSample_array(nbelems, samples);
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

void tfhe_bootstrap_FFT(LweSample *result, const LweBootstrappingKeyFFT *bk, Torus32 mu, const LweSample *x) {
    bootstrap_one(result, keys_of(bk), mu, x, true);
}

void tfhe_bootstrap_woKS_FFT(LweSample *result, const LweBootstrappingKeyFFT *bk, Torus32 mu, const LweSample *x) {
    bootstrap_one(result, keys_of(bk), mu, x, false);
}

// The coefficient-domain entry points (lwe-bootstrapping-functions.cpp:138-179) run the same GPU
// path on the same key: the reference computes their external products exactly with integer
// polynomial products, this library through its FFT (FP64 by default), so a result may differ
// from the reference's by a few Torus32 units while decrypting the same.
void tfhe_bootstrap(LweSample *result, const LweBootstrappingKey *bk, Torus32 mu, const LweSample *x) {
    bootstrap_one(result, keys_of(bk), mu, x, true);
}

void tfhe_bootstrap_woKS(LweSample *result, const LweBootstrappingKey *bk, Torus32 mu, const LweSample *x) {
    bootstrap_one(result, keys_of(bk), mu, x, false);
}

void tfhe_blindRotate_FFT(TLweSample *accum, const TGswSampleFFT *bk, const int32_t *bara, const int32_t n,
                          const TGswParams *bk_params) {
    if (n <= 0) return;
    int32_t first = 0;
    DropinKeys *k = own_fft_samples(bk, n, &first);
    ensure_on_device(k);
    const TLweParams *tp = bk_params->tlwe_params;
    blind_rotate_on(k->ck, k->stage, first, accum, bara, n, tp->k, tp->N);
}

void tfhe_blindRotateAndExtract_FFT(LweSample *result, const TorusPolynomial *v, const TGswSampleFFT *bk,
                                    const int32_t barb, const int32_t *bara, const int32_t n,
                                    const TGswParams *bk_params) {
    int32_t first = 0;
    DropinKeys *k = own_fft_samples(bk, n, &first);
    ensure_on_device(k);
    const TLweParams *tp = bk_params->tlwe_params;
    rotate_extract_on(k->ck, k->stage, first, result, v, barb, bara, n, tp->k, tp->N);
}

void tfhe_blindRotate(TLweSample *accum, const TGswSample *bk, const int32_t *bara, const int32_t n,
                      const TGswParams *bk_params) {
    if (n <= 0) return;
    const TLweParams *tp = bk_params->tlwe_params;
    DropinKeys *owner = nullptr;
    int32_t first = 0;
    if (own_coef_samples(bk, n, &owner, &first)) {
        ensure_on_device(owner);
        blind_rotate_on(owner->ck, owner->stage, first, accum, bara, n, tp->k, tp->N);
        return;
    }
    tfheb_cloud_key *ck = temporary_key(bk, n, bk_params);
    {
        StagingArea area;
        blind_rotate_on(ck, area, 0, accum, bara, n, tp->k, tp->N);
    }
    tfheb_cloud_key_free(ck);
}

void tfhe_blindRotateAndExtract(LweSample *result, const TorusPolynomial *v, const TGswSample *bk, const int32_t barb,
                                const int32_t *bara, const int32_t n, const TGswParams *bk_params) {
    const TLweParams *tp = bk_params->tlwe_params;
    DropinKeys *owner = nullptr;
    int32_t first = 0;
    if (own_coef_samples(bk, n, &owner, &first)) {
        ensure_on_device(owner);
        rotate_extract_on(owner->ck, owner->stage, first, result, v, barb, bara, n, tp->k, tp->N);
        return;
    }
    tfheb_cloud_key *ck = temporary_key(bk, n, bk_params);
    {
        StagingArea area;
        rotate_extract_on(ck, area, 0, result, v, barb, bara, n, tp->k, tp->N);
    }
    tfheb_cloud_key_free(ck);
}

void tGswExternProduct(TLweSample *result, const TGswSample *a, const TLweSample *b, const TGswParams *params) {
    extern_product(result, a, b, params, true);
}

void tGswExternMulToTLwe(TLweSample *accum, const TGswSample *sample, const TGswParams *params) {
    extern_product(accum, sample, accum, params, false);
}

// lweKeySwitch (lwe-keyswitch-functions.cpp:228-238) of one sample; the variance is the sum of the
// keyswitching-key rows' variances over the non-zero digits.
void lweKeySwitch(LweSample *result, const LweKeySwitchKey *ks, const LweSample *sample) {
    if (!ks || !ks->owner) die("keyswitching key is empty");
    DropinKeys *k = ks->owner;
    ensure_on_device(k);
    const int32_t n = k->p.n, kN = k->p.k * k->p.N;
    const size_t o_in = 0, o_out = kN + 1, o_terms = o_out + n + 1;
    Staged st(k->stage, k->ck, o_terms + 1);
    load_lwe(st.h(o_in), sample, kN);
    st.up(o_in, kN + 1);
    if (tfheb_keyswitch_device(k->ck, 1, st.d(o_in), st.d(o_out), nullptr) != TFHEB_OK ||
        tfheb_ks_terms_device(k->ck, 1, st.d(o_in), st.d(o_terms), nullptr) != TFHEB_OK)
        die("keyswitch");
    st.down(o_out, n + 2);
    st.finish("keyswitch");
    store_lwe(result, st.h(o_out), n);
    result->current_variance = ks_variance(k, *st.h(o_terms));
}

// ---- allocation of samples (polynomials.h:97-103, tlwe.h:222-235, lwesamples.h:70-83) ------------

TorusPolynomial *new_TorusPolynomial_array(int32_t nbelts, const int32_t N) {
    TorusPolynomial *p = alloc_array<TorusPolynomial>((size_t)nbelts);
    for (int32_t i = 0; i < nbelts; i++)
        put_bytes(&p[i], TorusPolynomial{N, static_cast<Torus32 *>(std::calloc((size_t)N, sizeof(Torus32)))});
    return p;
}
TorusPolynomial *new_TorusPolynomial(const int32_t N) { return new_TorusPolynomial_array(1, N); }
void delete_TorusPolynomial_array(int32_t nbelts, TorusPolynomial *obj) {
    if (!obj) return;
    for (int32_t i = 0; i < nbelts; i++) std::free(obj[i].coefsT);
    std::free(obj);
}
void delete_TorusPolynomial(TorusPolynomial *obj) { delete_TorusPolynomial_array(1, obj); }

TLweSample *new_TLweSample_array(int32_t nbelts, const TLweParams *params) {
    TLweSample *s = alloc_array<TLweSample>((size_t)nbelts);
    for (int32_t i = 0; i < nbelts; i++) {
        TorusPolynomial *a = new_TorusPolynomial_array(params->k + 1, params->N);
        put_bytes(&s[i], TLweSample{a, a + params->k, 0., params->k});
    }
    return s;
}
TLweSample *new_TLweSample(const TLweParams *params) { return new_TLweSample_array(1, params); }
void delete_TLweSample_array(int32_t nbelts, TLweSample *obj) {
    if (!obj) return;
    for (int32_t i = 0; i < nbelts; i++) delete_TorusPolynomial_array(obj[i].k + 1, obj[i].a);
    std::free(obj);
}
void delete_TLweSample(TLweSample *obj) { delete_TLweSample_array(1, obj); }

LweSample *new_LweSample_array(int32_t nbelts, const LweParams *params) {
    const int32_t n = params->n;
    LweSample *s = alloc_array<LweSample>((size_t)nbelts);
    for (int32_t i = 0; i < nbelts; i++) {
        s[i].a = static_cast<Torus32 *>(std::calloc((size_t)n, sizeof(Torus32)));
        s[i].b = 0;
        s[i].current_variance = 0.;
    }
    return s;
}
LweSample *new_LweSample(const LweParams *params) { return new_LweSample_array(1, params); }
void delete_LweSample_array(int32_t nbelts, LweSample *obj) {
    if (!obj) return;
    for (int32_t i = 0; i < nbelts; i++) std::free(obj[i].a);
    std::free(obj);
}
void delete_LweSample(LweSample *obj) { delete_LweSample_array(1, obj); }


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
    if (!ks->bkFFT || !keys_of(ks->bkFFT)->ck) die("cloud keyset has no key");
    if (!tfheb::io::write_cloud_content(F, keys_of(ks->bkFFT)->ck->ck)) die("writing a bootstrapping key");
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
