// engine.cu -- C-ABI entry points of libtfhe_b200.so (include/tfhe_b200.h): key lifecycle,
// device upload, and the batched gate pipeline
//     prologue -> blind rotation -> extraction -> keyswitch
// enqueued on one CUDA stream.  No CPU fallback: every gate runs through the kernels.
#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "internal.h"


namespace tfheb {

static thread_local std::string g_last_error;
std::atomic<int64_t> g_kernel_launches{0};
static std::atomic<int64_t> &g_launches = g_kernel_launches;

void set_error(const std::string &msg) { g_last_error = msg; }

static tfheb_status cuda_fail(cudaError_t e, const char *where) {
    set_error(std::string(where) + ": " + cudaGetErrorString(e));
    return e == cudaErrorMemoryAllocation ? TFHEB_ERR_NOMEM : TFHEB_ERR_CUDA;
}

#define TFHEB_CUDA(call)                                     \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call); \
    } while (0)

static bool valid_params(const tfheb_params *p) {
    if (!p) return false;
    if (p->n <= 0 || p->N <= 0 || p->k <= 0 || p->l <= 0 || p->Bgbit <= 0 || p->ks_t <= 0 || p->ks_basebit <= 0)
        return false;
    if ((p->N & (p->N - 1)) != 0) return false;
    if (p->l * p->Bgbit > 32 || p->ks_t * p->ks_basebit > 31) return false;
    return true;
}

template <typename T>
static tfheb_status grow(T *&ptr, size_t &cap, size_t need) {
    if (need <= cap) return TFHEB_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    TFHEB_CUDA(cudaMalloc((void **)&ptr, need * sizeof(T)));
    cap = need;
    return TFHEB_OK;
}

static int bara_stride_of(const tfheb_params &p) { return (p.n + 4) & ~3; }
int bara_stride_for(const tfheb_params &p) { return bara_stride_of(p); }

// gate linear combinations (boot-gates.cpp:34-319): constant numerator/denominator and weights
struct GateForm {
    int num, den, sa, sb;
};
static const GateForm kForms[10] = {
    {1, 8, -1, -1},  {1, 8, 1, 1},   {-1, 8, 1, 1},  {1, 4, 2, 2},  {-1, 4, -2, -2},
    {-1, 8, -1, -1}, {-1, 8, -1, 1}, {-1, 8, 1, -1}, {1, 8, -1, 1}, {1, 8, 1, -1},
};

void gate_form(int gate, int32_t *cst, int32_t *sa, int32_t *sb) {
    const GateForm &f = kForms[gate];
    *cst = modswitch_to_torus32(f.num, f.den);
    *sa = f.sa;
    *sb = f.sb;
}

// Builds bootstrap and gate descriptors for `count` gates with codes gates[g] (or one uniform code);
// gate g reads row g of each operand batch.
static void build_descs(int count, const int32_t *gates, int uniform, std::vector<BootDesc> &bd,
                        std::vector<GateDesc> &gd) {
    bd.clear();
    gd.assign(count, GateDesc{0, -1, 0});
    const int32_t mu8 = modswitch_to_torus32(1, 8);
    for (int g = 0; g < count; g++) {
        const int code = gates ? gates[g] : uniform;
        if (code == TFHEB_MUX) {
            const int32_t and_c = modswitch_to_torus32(-1, 8);
            gd[g].boot0 = (int32_t)bd.size();
            bd.push_back(BootDesc{g, and_c, 1, 1, 0, 1});   // (0,-1/8) + a + b
            gd[g].boot1 = (int32_t)bd.size();
            bd.push_back(BootDesc{g, and_c, -1, 1, 0, 2});  // (0,-1/8) - a + c
            gd[g].cst = mu8;                                // + (0, 1/8)
        } else {
            const GateForm &f = kForms[code];
            gd[g].boot0 = (int32_t)bd.size();
            bd.push_back(BootDesc{g, modswitch_to_torus32(f.num, f.den), (int8_t)f.sa, (int8_t)f.sb, 0, 1});
        }
    }
}

static tfheb_status ensure_device(CloudKey &ck, int precision) {
    if (ck.device < 0) {
        set_error("cloud key is not on a device (call tfheb_cloud_key_to_device)");
        return TFHEB_ERR_INVALID;
    }
    if (precision != TFHEB_FP64 && precision != TFHEB_SPLIT_FP32) {
        set_error("unknown precision");
        return TFHEB_ERR_INVALID;
    }
    if (!ck.dbsk[precision].bsk) {
        set_error("bootstrapping key not prepared for this precision");
        return TFHEB_ERR_INVALID;
    }
    if (!blind_rotate_supported(ck.p)) {
        set_error("no compiled blind-rotation kernel for this parameter set");
        return TFHEB_ERR_UNSUPPORTED;
    }
    TFHEB_CUDA(cudaSetDevice(ck.device));
    return TFHEB_OK;
}

tfheb_status prepare_device(CloudKey &ck, int precision) { return ensure_device(ck, precision); }

// Weight 2^S of the high limb in split mode.  The high-limb product sums must round to the exact
// integer.  Their FP32 error grows with
//   rms(product) = sqrt(N*(k+1)*l) * (2^Bgbit/sqrt12) * (2^(32-S)/sqrt12),
// so S is the smallest shift keeping rms(product) <= 2^18.  An FP32 model of the arithmetic then
// puts the error sigma at 0.021-0.028 of a unit for the reference's parameter sets, so a wrong
// rounding (an error above 1/2) is 18 or more sigma away.  Default parameters give S = 24, the
// N=2048 set S = 26, the 80-bit set S = 27.
int default_split_shift(const tfheb_params &p) {
    const double terms = std::sqrt((double)p.N * (p.k + 1) * p.l);
    const double digit_rms = std::ldexp(1.0, p.Bgbit) / std::sqrt(12.0);
    for (int S = 16; S <= 30; S++) {
        const double hi_rms = std::ldexp(1.0, 32 - S) / std::sqrt(12.0);
        if (terms * digit_rms * hi_rms <= 262144.0) return S;
    }
    return 30;
}


// Launch `fn` on stream s, bracketed by CUDA events when per-kernel profiling is on.
template <typename Fn>
static cudaError_t timed(CloudKey &ck, int which, cudaStream_t s, Fn &&fn) {
    if (!ck.prof) return fn();
    CloudKey::ProfRec r{which, nullptr, nullptr};
    cudaEventCreate(&r.a);
    cudaEventCreate(&r.b);
    cudaEventRecord(r.a, s);
    const cudaError_t e = fn();
    cudaEventRecord(r.b, s);
    ck.prof_pending.push_back(r);
    return e;
}

// Device pipeline for `count` gates described by (bd, gd) already uploaded.  d_terms (optional):
// per gate, the keyswitch's non-zero digit count.
static tfheb_status run_pipeline(CloudKey &ck, int precision, int count, int boots, const int32_t *d_a,
                                 const int32_t *d_b, const int32_t *d_c, int32_t *d_out, cudaStream_t s,
                                 int32_t *d_terms) {
    const tfheb_params &p = ck.p;
    const int bs = bara_stride_of(p);
    const int kN1 = p.k * p.N + 1;
    tfheb_status st;
    if ((st = grow(ck.d_bara, ck.bara_cap, (size_t)boots * bs)) != TFHEB_OK) return st;
    if ((st = grow(ck.d_acc, ck.acc_cap, (size_t)boots * (p.k + 1) * p.N)) != TFHEB_OK) return st;
    if ((st = grow(ck.d_ksin, ck.ksin_cap, (size_t)count * kN1)) != TFHEB_OK) return st;
    TFHEB_CUDA(timed(ck, 0, s, [&] { return launch_prologue(p, ck.d_bdesc, boots, d_a, d_b, d_c, ck.d_bara, bs, s); }));
    TFHEB_CUDA(timed(ck, 1, s, [&] {
        return launch_blind_rotate(p, precision, ck.dbsk[precision], ck.d_bara, bs, boots, p.n,
                                   modswitch_to_torus32(1, 8), nullptr, ck.d_acc, s, ck.d_err, ck.stall_producer,
                                   ck.wait_timeout_ns, ck.br[precision]);
    }));
    TFHEB_CUDA(timed(ck, 2, s, [&] { return launch_extract(p, ck.d_gdesc, count, ck.d_acc, ck.d_ksin, kN1, s); }));
    TFHEB_CUDA(timed(ck, 3, s, [&] {
        return launch_keyswitch(ck, count, ck.d_ksin, kN1, d_out, s);
    }));
    g_launches += 4;
    ck.launches += 4;
    if (d_terms) {
        TFHEB_CUDA(launch_ks_terms(p, count, ck.d_ksin, kN1, d_terms, s));
        g_launches += 1;
    }
    return TFHEB_OK;
}

// Reads and clears the key's device error word (after the stream has been synchronised).
tfheb_status check_device_error(CloudKey &ck) {
    int32_t err = 0;
    TFHEB_CUDA(cudaMemcpy(&err, ck.d_err, sizeof(err), cudaMemcpyDeviceToHost));
    if (err) {
        TFHEB_CUDA(cudaMemset(ck.d_err, 0, sizeof(err)));
        set_error("a bounded device-side wait expired (key stream stalled); results of that launch are invalid");
        return TFHEB_ERR_TIMEOUT;
    }
    return TFHEB_OK;
}

tfheb_status sync_key_stream(tfheb_cloud_key *c) {
    if (!c) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    if (ck.device < 0) return TFHEB_OK;
    TFHEB_CUDA(cudaSetDevice(ck.device));
    TFHEB_CUDA(cudaStreamSynchronize(ck.stream));
    return check_device_error(ck);
}

static tfheb_status upload_descs(CloudKey &ck, const std::vector<BootDesc> &bd, const std::vector<GateDesc> &gd,
                                 cudaStream_t s) {
    tfheb_status st;
    if ((st = grow(ck.d_bdesc, ck.bdesc_cap, bd.size())) != TFHEB_OK) return st;
    if ((st = grow(ck.d_gdesc, ck.gdesc_cap, gd.size())) != TFHEB_OK) return st;
    TFHEB_CUDA(cudaMemcpyAsync(ck.d_bdesc, bd.data(), bd.size() * sizeof(BootDesc), cudaMemcpyHostToDevice, s));
    TFHEB_CUDA(cudaMemcpyAsync(ck.d_gdesc, gd.data(), gd.size() * sizeof(GateDesc), cudaMemcpyHostToDevice, s));
    TFHEB_CUDA(cudaStreamSynchronize(s));  // host vectors are pageable temporaries
    return TFHEB_OK;
}

// A caller's buffer must be device (or managed) memory that the key's GPU can address: a host
// pointer or another GPU's memory would fault inside the kernels instead of returning an error.
tfheb_status check_device_ptr(const CloudKey &ck, const void *ptr, const char *what) {
    if (!ptr) return TFHEB_OK;
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, ptr) != cudaSuccess) {
        cudaGetLastError();
        set_error(std::string(what) + ": not a CUDA pointer");
        return TFHEB_ERR_INVALID;
    }
    if (attr.type == cudaMemoryTypeManaged) return TFHEB_OK;
    if (attr.type != cudaMemoryTypeDevice || attr.device != ck.device) {
        set_error(std::string(what) + ": not device memory on the key's GPU (device " + std::to_string(ck.device) + ")");
        return TFHEB_ERR_INVALID;
    }
    return TFHEB_OK;
}

// Calls that use the key's scratch (descriptors, rotation amounts, accumulators, extracted samples,
// host-batch copies) may come on different streams; each waits on the device for the previous one
// to finish with the scratch, then marks its own end, so they run in call order on the GPU.
static tfheb_status scratch_begin(CloudKey &ck, cudaStream_t s) {
    if (!ck.scratch_done) {
        TFHEB_CUDA(cudaEventCreateWithFlags(&ck.scratch_done, cudaEventDisableTiming));
        return TFHEB_OK;
    }
    TFHEB_CUDA(cudaStreamWaitEvent(s, ck.scratch_done, 0));
    return TFHEB_OK;
}
static tfheb_status scratch_end(CloudKey &ck, cudaStream_t s) {
    TFHEB_CUDA(cudaEventRecord(ck.scratch_done, s));
    return TFHEB_OK;
}

// Gate descriptors of `count` gates of one type.  They are per gate in batch order, so the array
// built for a count serves every smaller count of the same gate (a prefix); it is rebuilt only for
// another gate or a larger count.
static tfheb_status ensure_descs(CloudKey &ck, int gate, int count, cudaStream_t s) {
    if (ck.cached_gate == gate && count <= ck.cached_count) return TFHEB_OK;
    std::vector<BootDesc> bd;
    std::vector<GateDesc> gd;
    build_descs(count, nullptr, gate, bd, gd);
    const tfheb_status st = upload_descs(ck, bd, gd, s);
    if (st != TFHEB_OK) return st;
    ck.cached_gate = gate;
    ck.cached_count = count;
    return TFHEB_OK;
}

// `count` gates of one type on device buffers, enqueued on s (the key's lock held).  d_terms
// (optional, bootstrapped gates only): per gate, the keyswitch's non-zero digit count.
static tfheb_status gate_chunk(CloudKey &ck, int gate, int precision, int count, const int32_t *d_a,
                               const int32_t *d_b, const int32_t *d_c, int32_t *d_out, cudaStream_t s,
                               int32_t *d_terms = nullptr) {
    const int n1 = ck.p.n + 1;
    if (gate == TFHEB_COPY || gate == TFHEB_NOT) {
        // bootstrap-free (boot-gates.cpp:164-178)
        if (gate == TFHEB_COPY) {
            TFHEB_CUDA(cudaMemcpyAsync(d_out, d_a, (size_t)count * n1 * 4, cudaMemcpyDeviceToDevice, s));
            return TFHEB_OK;
        }
        TFHEB_CUDA(launch_negate(d_a, d_out, (size_t)count * n1, s));
        g_launches += 1;
        return TFHEB_OK;
    }
    if (!ck.dksk.rows) {
        set_error("the cloud key has no keyswitching key");
        return TFHEB_ERR_INVALID;
    }
    const tfheb_status st = ensure_descs(ck, gate, count, s);
    if (st != TFHEB_OK) return st;
    const int boots = gate == TFHEB_MUX ? 2 * count : count;
    return run_pipeline(ck, precision, count, boots, d_a, d_b, d_c, d_out, s, d_terms);
}

}  // namespace tfheb

using namespace tfheb;

extern "C" {

const char *tfheb_last_error(void) { return g_last_error.c_str(); }

int64_t tfheb_kernel_launches(void) { return g_launches.load(); }

tfheb_status tfheb_default_params(int32_t lambda, tfheb_params *out) {
    if (!out || lambda <= 0 || lambda > 128) {
        set_error("lambda must be in (0, 128] (80-bit and 128-bit sets)");
        return TFHEB_ERR_INVALID;
    }
    if (lambda > 80) *out = tfheb_params{630, 1024, 1, 3, 7, 8, 2, std::pow(2., -15), std::pow(2., -25)};
    else *out = tfheb_params{500, 1024, 1, 2, 10, 8, 2, 2.44e-5, 7.18e-9};
    return TFHEB_OK;
}

tfheb_status tfheb_large_params(tfheb_params *out) {
    if (!out) return TFHEB_ERR_INVALID;
    *out = tfheb_params{800, 2048, 1, 3, 8, 8, 2, std::pow(2., -15), std::pow(2., -25)};
    return TFHEB_OK;
}

tfheb_status tfheb_keygen(const tfheb_params *p, uint64_t seed, tfheb_secret_key **sk, tfheb_cloud_key **ck) {
    if (!valid_params(p) || !sk || !ck) {
        set_error("invalid parameters");
        return TFHEB_ERR_INVALID;
    }
    auto *s = new tfheb_secret_key();
    auto *c = new tfheb_cloud_key();
    keygen(*p, seed, s->sk, c->ck);
    *sk = s;
    *ck = c;
    return TFHEB_OK;
}

tfheb_status tfheb_cloud_key_import(const tfheb_params *p, const int32_t *bsk, const int32_t *ksk,
                                    tfheb_cloud_key **ck) {
    if (!valid_params(p) || !bsk || !ck) {
        set_error("invalid arguments");
        return TFHEB_ERR_INVALID;
    }
    auto *c = new tfheb_cloud_key();
    c->ck.p = *p;
    const size_t nb = (size_t)p->n * (p->k + 1) * p->l * (p->k + 1) * p->N;
    const size_t nk = (size_t)p->k * p->N * p->ks_t * (1 << p->ks_basebit) * (p->n + 1);
    c->ck.bsk_coef.assign(bsk, bsk + nb);
    if (ksk) c->ck.ksk.assign(ksk, ksk + nk);  // without one, the key serves blind rotations only
    *ck = c;
    return TFHEB_OK;
}

tfheb_status tfheb_secret_key_import(const tfheb_params *p, const int32_t *lwe_key, const int32_t *tlwe_key,
                                     tfheb_secret_key **sk) {
    if (!valid_params(p) || !lwe_key || !sk) {
        set_error("invalid arguments");
        return TFHEB_ERR_INVALID;
    }
    auto *s = new tfheb_secret_key();
    s->sk.p = *p;
    s->sk.lwe_key.assign(lwe_key, lwe_key + p->n);
    if (tlwe_key) s->sk.tlwe_key.assign(tlwe_key, tlwe_key + (size_t)p->k * p->N);
    *sk = s;
    return TFHEB_OK;
}

tfheb_status tfheb_secret_key_export(const tfheb_secret_key *sk, int32_t *lwe_key, int32_t *tlwe_key) {
    if (!sk) return TFHEB_ERR_INVALID;
    if (lwe_key) std::memcpy(lwe_key, sk->sk.lwe_key.data(), sk->sk.lwe_key.size() * 4);
    if (tlwe_key) std::memcpy(tlwe_key, sk->sk.tlwe_key.data(), sk->sk.tlwe_key.size() * 4);
    return TFHEB_OK;
}

tfheb_status tfheb_cloud_key_export(const tfheb_cloud_key *ck, int32_t *bsk, int32_t *ksk) {
    if (!ck) return TFHEB_ERR_INVALID;
    if (bsk) std::memcpy(bsk, ck->ck.bsk_coef.data(), ck->ck.bsk_coef.size() * 4);
    if (ksk) std::memcpy(ksk, ck->ck.ksk.data(), ck->ck.ksk.size() * 4);
    return TFHEB_OK;
}

tfheb_status tfheb_cloud_key_params(const tfheb_cloud_key *ck, tfheb_params *out) {
    if (!ck || !out) return TFHEB_ERR_INVALID;
    *out = ck->ck.p;
    return TFHEB_OK;
}

void tfheb_secret_key_free(tfheb_secret_key *sk) { delete sk; }

void tfheb_cloud_key_free(tfheb_cloud_key *c) {
    if (!c) return;
    CloudKey &ck = c->ck;
    if (ck.device >= 0) {
        cudaSetDevice(ck.device);
        for (auto &d : ck.dbsk) {
            cudaFree(d.bsk);
            cudaFree(d.tables);
            cudaFree(d.tables2);
        }
        free_keyswitch_key(ck.dksk);
        cudaFree(ck.d_bara);
        cudaFree(ck.d_acc);
        cudaFree(ck.d_ksin);
        cudaFree(ck.d_io);
        cudaFree(ck.d_terms);
        cudaFree(ck.d_bdesc);
        cudaFree(ck.d_gdesc);
        cudaFree(ck.d_err);
        if (ck.scratch_done) cudaEventDestroy(ck.scratch_done);
        if (ck.stream) cudaStreamDestroy(ck.stream);
    }
    delete c;
}

tfheb_status tfheb_encrypt(const tfheb_secret_key *sk, const int32_t *bits, int32_t count, uint64_t seed,
                           int32_t *out) {
    if (!sk || !bits || !out || count < 0) return TFHEB_ERR_INVALID;
    encrypt(sk->sk, bits, count, seed, out);
    return TFHEB_OK;
}

tfheb_status tfheb_encrypt_torus(const tfheb_secret_key *sk, const int32_t *mu, int32_t count, double stdev,
                                 uint64_t seed, int32_t *out) {
    if (!sk || count < 0 || (count > 0 && (!mu || !out)) || !(stdev >= 0)) return TFHEB_ERR_INVALID;
    encrypt_torus(sk->sk.p.n, sk->sk.lwe_key.data(), mu, count, stdev, seed, out);
    return TFHEB_OK;
}

tfheb_status tfheb_decrypt_torus(const tfheb_secret_key *sk, const int32_t *cts, int32_t count, int32_t msize,
                                 int32_t *out) {
    if (!sk || count < 0 || (count > 0 && (!cts || !out)) || msize < 1) return TFHEB_ERR_INVALID;
    const int n = sk->sk.p.n;
    for (int g = 0; g < count; g++) out[g] = approx_phase(phase(sk->sk, cts + (size_t)g * (n + 1)), msize);
    return TFHEB_OK;
}

tfheb_status tfheb_decrypt(const tfheb_secret_key *sk, const int32_t *cts, int32_t count, int32_t *bits,
                           int32_t *phases) {
    if (!sk || !cts || count < 0) return TFHEB_ERR_INVALID;
    const int n = sk->sk.p.n;
    for (int g = 0; g < count; g++) {
        const int32_t ph = phase(sk->sk, cts + (size_t)g * (n + 1));
        if (bits) bits[g] = ph > 0 ? 1 : 0;  // tfhe_gate_bootstrapping.cpp:162-165
        if (phases) phases[g] = ph;
    }
    return TFHEB_OK;
}

tfheb_status tfheb_cloud_key_to_device(tfheb_cloud_key *c, int32_t device, int32_t precision_mask,
                                       int32_t split_shift) {
    if (!c) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
        set_error("no CUDA device visible");
        return TFHEB_ERR_NO_DEVICE;
    }
    if (device < 0 || device >= ndev || (ck.device >= 0 && ck.device != device)) return TFHEB_ERR_INVALID;
    if (!blind_rotate_supported(ck.p)) {
        set_error("no compiled blind-rotation kernel for this parameter set");
        return TFHEB_ERR_UNSUPPORTED;
    }
    if (split_shift == 0) split_shift = default_split_shift(ck.p);
    if (split_shift < 8 || split_shift > 30) return TFHEB_ERR_INVALID;
    TFHEB_CUDA(cudaSetDevice(device));
    ck.device = device;
    if (!ck.stream) TFHEB_CUDA(cudaStreamCreateWithFlags(&ck.stream, cudaStreamNonBlocking));
    if (!ck.d_err) {
        TFHEB_CUDA(cudaMalloc((void **)&ck.d_err, sizeof(int32_t)));
        TFHEB_CUDA(cudaMemset(ck.d_err, 0, sizeof(int32_t)));
    }
    const tfheb_params &p = ck.p;
    // keyswitching key in the layouts of the keyswitch kernels (absent from keys made for blind
    // rotations only)
    if (!ck.ksk.empty()) TFHEB_CUDA(upload_keyswitch_key(ck));
    std::vector<double> tab;
    build_tables_fp64(p.N, tab);
    // the FFT-domain keys are computed on the device (key_transform.cu) from the coefficient key
    // and the FP64 tables, both staged in temporary device buffers freed on every return path
    struct Temp {
        void *p = nullptr;
        ~Temp() {
            if (p) cudaFree(p);
        }
    } d_coef, d_tab64;
    const size_t polys = (size_t)p.n * (p.k + 1) * p.l * (p.k + 1);
    for (int prec = 0; prec < 2; prec++) {
        if (!(precision_mask & (1 << prec))) continue;
        DeviceBsk &d = ck.dbsk[prec];
        if (d.bsk && (prec == TFHEB_FP64 || d.split_shift == split_shift)) continue;
        if (d.bsk) {
            cudaFree(d.bsk);
            cudaFree(d.tables);
            cudaFree(d.tables2);
            d.bsk = d.tables = d.tables2 = nullptr;
        }
        if (!d_coef.p) {
            TFHEB_CUDA(cudaMalloc(&d_coef.p, ck.bsk_coef.size() * sizeof(int32_t)));
            TFHEB_CUDA(cudaMemcpy(d_coef.p, ck.bsk_coef.data(), ck.bsk_coef.size() * sizeof(int32_t),
                                  cudaMemcpyHostToDevice));
            TFHEB_CUDA(cudaMalloc(&d_tab64.p, tab.size() * sizeof(double)));
            TFHEB_CUDA(cudaMemcpy(d_tab64.p, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice));
        }
        d.bsk_bytes = polys * (size_t)(p.N / 2) * 16;
        TFHEB_CUDA(cudaMalloc(&d.bsk, d.bsk_bytes));
        d.split_shift = prec == TFHEB_SPLIT_FP32 ? split_shift : 0;
        TFHEB_CUDA(launch_bsk_to_fft(p, prec, static_cast<const int32_t *>(d_coef.p),
                                     static_cast<const double *>(d_tab64.p), d.bsk, split_shift, ck.stream));
        if (prec == TFHEB_FP64) {
            TFHEB_CUDA(cudaMalloc(&d.tables, tab.size() * sizeof(double)));
            TFHEB_CUDA(cudaMemcpy(d.tables, tab.data(), tab.size() * sizeof(double), cudaMemcpyHostToDevice));
        } else {
            std::vector<float> tf;
            build_tables_f32(p.N, tf);
            TFHEB_CUDA(cudaMalloc(&d.tables, tf.size() * sizeof(float)));
            TFHEB_CUDA(cudaMemcpy(d.tables, tf.data(), tf.size() * sizeof(float), cudaMemcpyHostToDevice));
            build_tables_f32_paired(p.N, tf);
            TFHEB_CUDA(cudaMalloc(&d.tables2, tf.size() * sizeof(float)));
            TFHEB_CUDA(cudaMemcpy(d.tables2, tf.data(), tf.size() * sizeof(float), cudaMemcpyHostToDevice));
        }
    }
    TFHEB_CUDA(cudaStreamSynchronize(ck.stream));
    return TFHEB_OK;
}

/* Inspection of the device FFT-domain key (layouts in key_transform.cu). */
tfheb_status tfheb_cloud_key_fft_download(const tfheb_cloud_key *c, int32_t precision, void *out, size_t bytes) {
    if (!c || !out || (precision != TFHEB_FP64 && precision != TFHEB_SPLIT_FP32)) return TFHEB_ERR_INVALID;
    const DeviceBsk &d = c->ck.dbsk[precision];
    if (!d.bsk) {
        set_error("tfheb_cloud_key_fft_download: no FFT-domain key of that precision on the device");
        return TFHEB_ERR_INVALID;
    }
    if (bytes != d.bsk_bytes) {
        set_error("tfheb_cloud_key_fft_download: buffer size must be " + std::to_string(d.bsk_bytes) + " bytes");
        return TFHEB_ERR_INVALID;
    }
    TFHEB_CUDA(cudaSetDevice(c->ck.device));
    TFHEB_CUDA(cudaMemcpy(out, d.bsk, bytes, cudaMemcpyDeviceToHost));
    return TFHEB_OK;
}

tfheb_status tfheb_gate_batch_device(tfheb_cloud_key *c, int32_t gate, int32_t precision, int32_t count,
                                     const int32_t *d_a, const int32_t *d_b, const int32_t *d_c, int32_t *d_out,
                                     void *stream) {
    if (!c || count < 0 || gate < 0 || gate > TFHEB_COPY) return TFHEB_ERR_INVALID;
    if (count > 0 && (!d_a || !d_out || (gate == TFHEB_MUX && (!d_b || !d_c)) || (gate < TFHEB_MUX && !d_b)))
        return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    tfheb_status st = ensure_device(ck, precision);
    if (st != TFHEB_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : ck.stream;
    if (count == 0) return TFHEB_OK;
    for (auto [ptr, what] : {std::pair<const void *, const char *>{d_a, "d_a"}, {d_b, "d_b"}, {d_c, "d_c"}, {d_out, "d_out"}})
        if ((st = check_device_ptr(ck, ptr, what)) != TFHEB_OK) return st;
    if ((st = scratch_begin(ck, s)) != TFHEB_OK) return st;
    st = gate_chunk(ck, gate, precision, count, d_a, d_b, d_c, d_out, s);
    const tfheb_status se = scratch_end(ck, s);
    return st != TFHEB_OK ? st : se;
}

// Host buffers: inputs in, one launch sequence over the whole batch, output back, on the key's
// stream.  Splitting a batch into wave-sized chunks whose copies overlap the neighbouring chunks'
// gates gained nothing on B200 (102.4k NAND/s at 4096 split-FP32 gates, against 102.3k-103.9k
// unsplit across boxes): the copies it hides (about 0.6 ms per 4096 gates) are offset by what the
// chunks add, a keyswitch per chunk that streams the keyswitching key through L2 again and evicts
// part of the bootstrapping key, and a ramp and tail per blind-rotation launch.
static tfheb_status gate_batch_host(tfheb_cloud_key *c, int32_t gate, int32_t precision, int32_t count,
                                    const int32_t *a, const int32_t *b, const int32_t *cc, int32_t *out,
                                    int32_t *terms) {
    if (!c || count < 0 || gate < 0 || gate > TFHEB_COPY) return TFHEB_ERR_INVALID;
    if (count == 0) return TFHEB_OK;
    if (!a || !out || (gate == TFHEB_MUX && (!b || !cc)) || (gate < TFHEB_MUX && !b)) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    tfheb_status st = ensure_device(ck, precision);
    if (st != TFHEB_OK) return st;
    const size_t sz = (size_t)count * (ck.p.n + 1);
    if ((st = grow(ck.d_io, ck.io_cap, 4 * sz)) != TFHEB_OK) return st;
    const bool with_terms = terms && gate != TFHEB_NOT && gate != TFHEB_COPY;
    if (terms && !with_terms)
        for (int32_t g = 0; g < count; g++) terms[g] = -1;  // no keyswitch: the input's variance carries over
    if (with_terms && (st = grow(ck.d_terms, ck.terms_cap, (size_t)count)) != TFHEB_OK) return st;
    int32_t *dio = ck.d_io;
    cudaStream_t s = ck.stream;
    if ((st = scratch_begin(ck, s)) != TFHEB_OK) return st;
    TFHEB_CUDA(cudaMemcpyAsync(dio, a, sz * 4, cudaMemcpyHostToDevice, s));
    if (b) TFHEB_CUDA(cudaMemcpyAsync(dio + sz, b, sz * 4, cudaMemcpyHostToDevice, s));
    if (cc) TFHEB_CUDA(cudaMemcpyAsync(dio + 2 * sz, cc, sz * 4, cudaMemcpyHostToDevice, s));
    st = gate_chunk(ck, gate, precision, count, dio, b ? dio + sz : nullptr, cc ? dio + 2 * sz : nullptr,
                    dio + 3 * sz, s, with_terms ? ck.d_terms : nullptr);
    if (st == TFHEB_OK) TFHEB_CUDA(cudaMemcpyAsync(out, dio + 3 * sz, sz * 4, cudaMemcpyDeviceToHost, s));
    if (st == TFHEB_OK && with_terms)
        TFHEB_CUDA(cudaMemcpyAsync(terms, ck.d_terms, (size_t)count * 4, cudaMemcpyDeviceToHost, s));
    if (st == TFHEB_OK) st = scratch_end(ck, s);
    const cudaError_t e = cudaStreamSynchronize(s);  // drain, also after an error
    if (st != TFHEB_OK) return st;
    TFHEB_CUDA(e);
    return check_device_error(ck);
}

tfheb_status tfheb_gate_batch(tfheb_cloud_key *c, int32_t gate, int32_t precision, int32_t count,
                              const int32_t *a, const int32_t *b, const int32_t *cc, int32_t *out) {
    return gate_batch_host(c, gate, precision, count, a, b, cc, out, nullptr);
}

tfheb_status tfheb_gate_batch_terms(tfheb_cloud_key *c, int32_t gate, int32_t precision, int32_t count,
                                    const int32_t *a, const int32_t *b, const int32_t *cc, int32_t *out,
                                    int32_t *terms) {
    if (!terms) return TFHEB_ERR_INVALID;
    return gate_batch_host(c, gate, precision, count, a, b, cc, out, terms);
}

// Bootstraps without keyswitch of `count` samples (the key's lock held).
static tfheb_status bootstrap_woks_locked(CloudKey &ck, int32_t precision, int32_t mu, int32_t count,
                                          const int32_t *d_in, int32_t *d_out, cudaStream_t s) {
    const tfheb_params &p = ck.p;
    // identity combination: x = in, one bootstrap per sample, no MUX term
    std::vector<BootDesc> bd(count);
    std::vector<GateDesc> gd(count);
    for (int g = 0; g < count; g++) {
        bd[g] = BootDesc{g, 0, 1, 0, 0, 0};
        gd[g] = GateDesc{g, -1, 0};
    }
    tfheb_status st;
    if ((st = upload_descs(ck, bd, gd, s)) != TFHEB_OK) return st;
    ck.cached_gate = ck.cached_count = -1;
    const int bs = bara_stride_of(p);
    if ((st = grow(ck.d_bara, ck.bara_cap, (size_t)count * bs)) != TFHEB_OK) return st;
    if ((st = grow(ck.d_acc, ck.acc_cap, (size_t)count * (p.k + 1) * p.N)) != TFHEB_OK) return st;
    TFHEB_CUDA(launch_prologue(p, ck.d_bdesc, count, d_in, d_in, d_in, ck.d_bara, bs, s));
    TFHEB_CUDA(launch_blind_rotate(p, precision, ck.dbsk[precision], ck.d_bara, bs, count, p.n, mu, nullptr,
                                   ck.d_acc, s, ck.d_err, ck.stall_producer, ck.wait_timeout_ns,
                                   ck.br[precision]));
    TFHEB_CUDA(launch_extract(p, ck.d_gdesc, count, ck.d_acc, d_out, p.k * p.N + 1, s));
    g_launches += 3;
    return TFHEB_OK;
}

tfheb_status tfheb_bootstrap_woks_device(tfheb_cloud_key *c, int32_t precision, int32_t mu, int32_t count,
                                         const int32_t *d_in, int32_t *d_out, void *stream) {
    if (!c || count < 0 || !d_in || !d_out) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    tfheb_status st = ensure_device(ck, precision);
    if (st != TFHEB_OK) return st;
    if (count == 0) return TFHEB_OK;
    if ((st = check_device_ptr(ck, d_in, "d_in")) != TFHEB_OK || (st = check_device_ptr(ck, d_out, "d_out")) != TFHEB_OK)
        return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : ck.stream;
    if ((st = scratch_begin(ck, s)) != TFHEB_OK) return st;
    st = bootstrap_woks_locked(ck, precision, mu, count, d_in, d_out, s);
    const tfheb_status se = scratch_end(ck, s);
    return st != TFHEB_OK ? st : se;
}

// Bootstrap then keyswitch, under one hold of the key's lock: the intermediate samples live in the
// key's scratch, which another call on the key could otherwise reallocate in between.
tfheb_status tfheb_bootstrap_device(tfheb_cloud_key *c, int32_t precision, int32_t mu, int32_t count,
                                    const int32_t *d_in, int32_t *d_out, void *stream) {
    if (!c || count < 0 || !d_in || !d_out) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    tfheb_status st = ensure_device(ck, precision);
    if (st != TFHEB_OK) return st;
    if (!ck.dksk.rows) {
        set_error("the cloud key has no keyswitching key");
        return TFHEB_ERR_INVALID;
    }
    if (count == 0) return TFHEB_OK;
    if ((st = check_device_ptr(ck, d_in, "d_in")) != TFHEB_OK || (st = check_device_ptr(ck, d_out, "d_out")) != TFHEB_OK)
        return st;
    if ((st = grow(ck.d_ksin, ck.ksin_cap, (size_t)count * (ck.p.k * ck.p.N + 1))) != TFHEB_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : ck.stream;
    if ((st = scratch_begin(ck, s)) != TFHEB_OK) return st;
    st = bootstrap_woks_locked(ck, precision, mu, count, d_in, ck.d_ksin, s);
    if (st == TFHEB_OK) {
        const cudaError_t e = launch_keyswitch(ck, count, ck.d_ksin, ck.p.k * ck.p.N + 1, d_out, s);
        if (e != cudaSuccess) st = cuda_fail(e, "launch_keyswitch");
        g_launches += 1;
    }
    const tfheb_status se = scratch_end(ck, s);
    return st != TFHEB_OK ? st : se;
}

// The device key from TGSW step `first` on: every step's rows are contiguous in both layouts.
static DeviceBsk key_from_step(const CloudKey &ck, int precision, int first) {
    DeviceBsk d = ck.dbsk[precision];
    const tfheb_params &p = ck.p;
    const size_t step_bytes = (size_t)(p.k + 1) * p.l * (p.k + 1) * (p.N / 2) * 16;
    d.bsk = static_cast<unsigned char *>(d.bsk) + step_bytes * (size_t)first;
    return d;
}

tfheb_status tfheb_blind_rotate_steps_device(tfheb_cloud_key *c, int32_t precision, int32_t count, int32_t first_step,
                                             int32_t nsteps, const int32_t *d_bara, int32_t *d_acc, void *stream) {
    if (!c || count < 0 || !d_bara || !d_acc || nsteps < 0 || first_step < 0) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    if ((int64_t)first_step + nsteps > ck.p.n) {
        set_error("blind rotation: steps beyond the key's " + std::to_string(ck.p.n) + " TGSW samples");
        return TFHEB_ERR_INVALID;
    }
    tfheb_status st = ensure_device(ck, precision);
    if (st != TFHEB_OK) return st;
    if (count == 0 || nsteps == 0) return TFHEB_OK;
    if ((st = check_device_ptr(ck, d_bara, "d_bara")) != TFHEB_OK || (st = check_device_ptr(ck, d_acc, "d_acc")) != TFHEB_OK)
        return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : ck.stream;
    // in place: acc_in == acc_out is safe (each team reads its row fully before writing it back)
    TFHEB_CUDA(launch_blind_rotate(ck.p, precision, key_from_step(ck, precision, first_step), d_bara, nsteps, count,
                                   nsteps, 0, d_acc, d_acc, s, ck.d_err, ck.stall_producer, ck.wait_timeout_ns,
                                   ck.br[precision]));
    g_launches += 1;
    return TFHEB_OK;
}

tfheb_status tfheb_blind_rotate_device(tfheb_cloud_key *c, int32_t precision, int32_t count, int32_t nsteps,
                                       const int32_t *d_bara, int32_t *d_acc, void *stream) {
    return tfheb_blind_rotate_steps_device(c, precision, count, 0, nsteps, d_bara, d_acc, stream);
}

tfheb_status tfheb_blind_rotate_extract_device(tfheb_cloud_key *c, int32_t precision, int32_t count,
                                               int32_t first_step, int32_t nsteps, const int32_t *d_v,
                                               const int32_t *d_barb, const int32_t *d_bara, int32_t *d_out,
                                               void *stream) {
    if (!c || count < 0 || nsteps < 0 || first_step < 0) return TFHEB_ERR_INVALID;
    if (count > 0 && (!d_v || !d_barb || !d_out || (nsteps > 0 && !d_bara))) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    const tfheb_params &p = ck.p;
    if ((int64_t)first_step + nsteps > p.n) {
        set_error("blind rotation: steps beyond the key's " + std::to_string(p.n) + " TGSW samples");
        return TFHEB_ERR_INVALID;
    }
    tfheb_status st = ensure_device(ck, precision);
    if (st != TFHEB_OK) return st;
    if (count == 0) return TFHEB_OK;
    for (auto [ptr, what] : {std::pair<const void *, const char *>{d_v, "d_v"}, {d_barb, "d_barb"}, {d_bara, "d_bara"},
                             {d_out, "d_out"}})
        if ((st = check_device_ptr(ck, ptr, what)) != TFHEB_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : ck.stream;
    if ((st = scratch_begin(ck, s)) != TFHEB_OK) return st;
    if ((st = grow(ck.d_acc, ck.acc_cap, (size_t)count * (p.k + 1) * p.N)) == TFHEB_OK) {
        cudaError_t e = launch_testvec(p, count, d_v, d_barb, ck.d_acc, s);
        if (e == cudaSuccess && nsteps > 0)
            e = launch_blind_rotate(p, precision, key_from_step(ck, precision, first_step), d_bara, nsteps, count,
                                    nsteps, 0, ck.d_acc, ck.d_acc, s, ck.d_err, ck.stall_producer,
                                    ck.wait_timeout_ns, ck.br[precision]);
        if (e == cudaSuccess) e = launch_extract(p, nullptr, count, ck.d_acc, d_out, p.k * p.N + 1, s);
        if (e != cudaSuccess) st = cuda_fail(e, "tfheb_blind_rotate_extract_device");
        g_launches += nsteps > 0 ? 3 : 2;
    }
    const tfheb_status se = scratch_end(ck, s);
    return st != TFHEB_OK ? st : se;
}

tfheb_status tfheb_extern_product_device(tfheb_cloud_key *c, int32_t precision, int32_t count, int32_t step,
                                         const int32_t *d_in, int32_t *d_out, void *stream) {
    if (!c || count < 0 || step < 0) return TFHEB_ERR_INVALID;
    if (count > 0 && (!d_in || !d_out)) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    if (step >= ck.p.n) {
        set_error("external product: the key has " + std::to_string(ck.p.n) + " TGSW samples");
        return TFHEB_ERR_INVALID;
    }
    tfheb_status st = ensure_device(ck, precision);
    if (st != TFHEB_OK) return st;
    if (count == 0) return TFHEB_OK;
    if ((st = check_device_ptr(ck, d_in, "d_in")) != TFHEB_OK || (st = check_device_ptr(ck, d_out, "d_out")) != TFHEB_OK)
        return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : ck.stream;
    const cudaError_t e = launch_extern_product(ck.p, precision, key_from_step(ck, precision, step), count, d_in, d_out,
                                                s, ck.d_err, ck.wait_timeout_ns);
    if (e == cudaErrorInvalidValue) {
        set_error("external product: no compiled kernel for this ring degree and gadget length");
        return TFHEB_ERR_UNSUPPORTED;
    }
    TFHEB_CUDA(e);
    g_launches += 1;
    return TFHEB_OK;
}

tfheb_status tfheb_ks_terms_device(tfheb_cloud_key *c, int32_t count, const int32_t *d_in, int32_t *d_terms,
                                   void *stream) {
    if (!c || count < 0 || (count > 0 && (!d_in || !d_terms))) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    if (ck.device < 0) {
        set_error("cloud key is not on a device (call tfheb_cloud_key_to_device)");
        return TFHEB_ERR_INVALID;
    }
    TFHEB_CUDA(cudaSetDevice(ck.device));
    if (count == 0) return TFHEB_OK;
    tfheb_status st;
    if ((st = check_device_ptr(ck, d_in, "d_in")) != TFHEB_OK || (st = check_device_ptr(ck, d_terms, "d_terms")) != TFHEB_OK)
        return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : ck.stream;
    TFHEB_CUDA(launch_ks_terms(ck.p, count, d_in, ck.p.k * ck.p.N + 1, d_terms, s));
    g_launches += 1;
    return TFHEB_OK;
}

tfheb_status tfheb_keyswitch_device(tfheb_cloud_key *c, int32_t count, const int32_t *d_in, int32_t *d_out,
                                    void *stream) {
    if (!c || count < 0 || !d_in || !d_out) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    if (ck.device < 0 || !ck.dksk.rows) {
        set_error("the cloud key has no keyswitching key on a device");
        return TFHEB_ERR_INVALID;
    }
    TFHEB_CUDA(cudaSetDevice(ck.device));
    if (count == 0) return TFHEB_OK;
    tfheb_status st;
    if ((st = check_device_ptr(ck, d_in, "d_in")) != TFHEB_OK || (st = check_device_ptr(ck, d_out, "d_out")) != TFHEB_OK)
        return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : ck.stream;
    TFHEB_CUDA(launch_keyswitch(ck, count, d_in, ck.p.k * ck.p.N + 1, d_out, s));
    g_launches += 1;
    return TFHEB_OK;
}

tfheb_status tfheb_synchronize(tfheb_cloud_key *c) {
    if (!c) return TFHEB_ERR_INVALID;
    CloudKey &ck = c->ck;
    if (ck.device < 0) return TFHEB_OK;
    TFHEB_CUDA(cudaSetDevice(ck.device));
    TFHEB_CUDA(cudaStreamSynchronize(ck.stream));
    TFHEB_CUDA(cudaDeviceSynchronize());
    TFHEB_CUDA(cudaGetLastError());
    return check_device_error(ck);
}

tfheb_status tfheb_set_wait_timeout(tfheb_cloud_key *c, uint64_t timeout_ns) {
    if (!c || timeout_ns == 0) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    c->ck.wait_timeout_ns = timeout_ns;
    return TFHEB_OK;
}

tfheb_status tfheb_br_variants(int32_t N, int32_t precision, int32_t *teams_per_cta, int32_t *ring_depth,
                               int32_t cap, int32_t *count) {
    if (!count) return TFHEB_ERR_INVALID;
    *count = br_variants(N, 3, precision, teams_per_cta, ring_depth, cap);
    return TFHEB_OK;
}

tfheb_status tfheb_cloud_key_br_variants(const tfheb_cloud_key *c, int32_t precision, int32_t *teams_per_cta,
                                         int32_t *ring_depth, int32_t cap, int32_t *count) {
    if (!c || !count || cap < 0) return TFHEB_ERR_INVALID;
    *count = br_variants(c->ck.p.N, c->ck.p.l, precision, teams_per_cta, ring_depth, cap);
    return TFHEB_OK;
}

tfheb_status tfheb_cloud_key_br_plans(const tfheb_cloud_key *c, int32_t precision, int32_t *plan, int32_t cap,
                                      int32_t *count) {
    if (!c || !count || cap < 0) return TFHEB_ERR_INVALID;
    *count = br_variant_plans(c->ck.p.N, c->ck.p.l, precision, plan, cap);
    return TFHEB_OK;
}

tfheb_status tfheb_set_br_variant(tfheb_cloud_key *c, int32_t precision, int32_t variant) {
    if (!c || (precision != TFHEB_FP64 && precision != TFHEB_SPLIT_FP32)) return TFHEB_ERR_INVALID;
    if (variant < 0 || variant >= br_variants(c->ck.p.N, c->ck.p.l, precision, nullptr, nullptr, 0))
        return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    c->ck.br[precision].tuned = variant;
    return TFHEB_OK;
}

tfheb_status tfheb_set_keyswitch_kernel(tfheb_cloud_key *c, int32_t which) {
    if (!c || which < 0 || which > 4) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    const tfheb_params &p = c->ck.p;
    if (which >= 2 && !(p.ks_t == 8 && p.ks_basebit == 2)) {
        set_error("tfheb_set_keyswitch_kernel: no tiled keyswitch for this parameter set");
        return TFHEB_ERR_UNSUPPORTED;
    }
    c->ck.ks_kernel = which;
    return TFHEB_OK;
}

// Times every compiled blind-rotation variant on `boots` synthetic bootstraps (random rotation
// amounts, the key's own bootstrapping key) and keeps the fastest for this key and precision.
// Device time of one blind-rotation launch of compiled variant g over `boots` bootstraps (the second
// of two runs; the first warms up).
static tfheb_status time_variant(CloudKey &ck, int precision, int g, int boots, cudaEvent_t e0, cudaEvent_t e1,
                                 float *ms) {
    const tfheb_params &p = ck.p;
    for (int rep = 0; rep < 2; rep++) {
        TFHEB_CUDA(cudaEventRecord(e0, ck.stream));
        TFHEB_CUDA(launch_blind_rotate_exact(p, precision, ck.dbsk[precision], ck.d_bara, bara_stride_of(p), boots, p.n,
                                             modswitch_to_torus32(1, 8), nullptr, ck.d_acc, ck.stream, ck.d_err, 0,
                                             ck.wait_timeout_ns, g));
        TFHEB_CUDA(cudaEventRecord(e1, ck.stream));
        TFHEB_CUDA(cudaEventSynchronize(e1));
        TFHEB_CUDA(cudaEventElapsedTime(ms, e0, e1));
    }
    return TFHEB_OK;
}

// Times every tuned variant on `boots` synthetic bootstraps and keeps the fastest.  Then, for each
// bootstraps-per-CTA need g below the winner's G, times every compiled variant with g <= G <= the
// winner's on one full wave (SMs x g bootstraps) and records the fastest in the key's small-batch
// table (BrChoice).
tfheb_status tfheb_autotune(tfheb_cloud_key *c, int32_t precision, int32_t boots, double *ms_out, int32_t cap) {
    if (!c || boots <= 0) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    tfheb_status st = ensure_device(ck, precision);
    if (st != TFHEB_OK) return st;
    const tfheb_params &p = ck.p;
    const int bs = bara_stride_of(p);
    int sms = 0;
    TFHEB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ck.device));
    const int most = std::max(boots, sms * (kSmallNeeds - 1));
    if ((st = grow(ck.d_bara, ck.bara_cap, (size_t)most * bs)) != TFHEB_OK) return st;
    if ((st = grow(ck.d_acc, ck.acc_cap, (size_t)most * (p.k + 1) * p.N)) != TFHEB_OK) return st;
    std::vector<int32_t> bara((size_t)most * bs);
    uint64_t x = 0x9E3779B97F4A7C15ull;
    for (auto &v : bara) {
        x ^= x << 13; x ^= x >> 7; x ^= x << 17;
        v = (int32_t)(x % (uint64_t)(2 * p.N));
    }
    TFHEB_CUDA(cudaMemcpy(ck.d_bara, bara.data(), bara.size() * 4, cudaMemcpyHostToDevice));
    struct Events {
        cudaEvent_t a = nullptr, b = nullptr;
        ~Events() {
            if (a) cudaEventDestroy(a);
            if (b) cudaEventDestroy(b);
        }
    } ev;
    TFHEB_CUDA(cudaEventCreate(&ev.a));
    TFHEB_CUDA(cudaEventCreate(&ev.b));
    const int nv = br_variants(p.N, p.l, precision, nullptr, nullptr, 0);
    int best = 0;
    float best_ms = 1e30f;
    for (int v = 0; v < nv; v++) {
        float ms = 0;
        if ((st = time_variant(ck, precision, br_tuned_global(p.N, p.l, precision, v), boots, ev.a, ev.b, &ms)) != TFHEB_OK)
            return st;
        if (ms_out && v < cap) ms_out[v] = ms;
        if (ms < best_ms) {
            best_ms = ms;
            best = v;
        }
    }
    BrChoice choice;
    choice.tuned = best;
    const int best_g = br_tuned_global(p.N, p.l, precision, best);
    int best_G = 0;
    br_variant_info(best_g, nullptr, nullptr, nullptr, &best_G, nullptr, nullptr);
    for (int need = 1; need < best_G && need < kSmallNeeds; need++) {
        float fastest = 1e30f;
        for (int g = 0; g < br_variant_count(); g++) {
            int N = 0, l = 0, prec = 0, G = 0;
            br_variant_info(g, &N, &l, &prec, &G, nullptr, nullptr);
            if (N != p.N || l != p.l || prec != precision || G < need || G > best_G) continue;
            float ms = 0;
            if ((st = time_variant(ck, precision, g, sms * need, ev.a, ev.b, &ms)) != TFHEB_OK) return st;
            if (ms < fastest) {
                fastest = ms;
                choice.small[need] = g == best_g ? -1 : g;
            }
        }
    }
    if ((st = check_device_error(ck)) != TFHEB_OK) return st;
    ck.br[precision] = choice;
    return TFHEB_OK;
}

tfheb_status tfheb_test_stall_key_stream(tfheb_cloud_key *c, int32_t stall) {
    if (!c) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    c->ck.stall_producer = stall != 0;
    return TFHEB_OK;
}

tfheb_status tfheb_profile(tfheb_cloud_key *c, int32_t enable) {
    if (!c) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    c->ck.prof = enable != 0;
    return TFHEB_OK;
}

tfheb_status tfheb_profile_read(tfheb_cloud_key *c, double *ms, int64_t *launches, int32_t reset) {
    if (!c) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    for (auto &r : ck.prof_pending) {
        float t = 0;
        cudaEventSynchronize(r.b);
        cudaEventElapsedTime(&t, r.a, r.b);
        ck.prof_ms[r.which] += t;
        ck.prof_n[r.which] += 1;
        cudaEventDestroy(r.a);
        cudaEventDestroy(r.b);
    }
    ck.prof_pending.clear();
    for (int i = 0; i < 4; i++) {
        if (ms) ms[i] = ck.prof_ms[i];
        if (launches) launches[i] = ck.prof_n[i];
        if (reset) {
            ck.prof_ms[i] = 0;
            ck.prof_n[i] = 0;
        }
    }
    return TFHEB_OK;
}

tfheb_status tfheb_measure_fma_peak(int32_t device, int32_t precision, double *tflops) {
    if (!tflops || (precision != TFHEB_FP64 && precision != TFHEB_SPLIT_FP32)) return TFHEB_ERR_INVALID;
    TFHEB_CUDA(cudaSetDevice(device));
    TFHEB_CUDA(measure_fma_peak(precision, tflops));
    return TFHEB_OK;
}

int32_t tfheb_default_split_shift(const tfheb_params *p) { return p ? default_split_shift(*p) : 0; }

tfheb_status tfheb_fft_slot_order(int32_t N, int32_t *slot_freq) {
    std::vector<int32_t> sf;
    fill_slot_freq(N, sf);
    if (sf.empty() || !slot_freq) return TFHEB_ERR_UNSUPPORTED;
    std::memcpy(slot_freq, sf.data(), sf.size() * 4);
    return TFHEB_OK;
}

}  // extern "C"
