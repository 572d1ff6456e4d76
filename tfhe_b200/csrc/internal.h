// internal.h -- shared declarations of the tfhe_b200 engine (host runtime + kernel launchers).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/tfhe_b200.h"

namespace tfheb {

constexpr int kR = 8;  // FFT points per thread

// Per-bootstrap descriptor: which inputs the gate's linear combination reads and with what weights
// (boot-gates.cpp:34-370).  x/y select the operand: 0 = a, 1 = b, 2 = c.
struct BootDesc {
    int32_t gate;  // gate (output) index
    int32_t cst;   // Torus32 constant added to b
    int8_t sa, sb; // integer weights of operands x and y
    uint8_t xsel, ysel;
};

// Per-gate descriptor for the extraction stage: output = extract(acc[boot0]) (+ extract(acc[boot1]))
// + (0, cst).  boot1 < 0 for one-bootstrap gates.
struct GateDesc {
    int32_t boot0, boot1;
    int32_t cst;
};

// Device-side FFT-domain bootstrapping key and tables for one precision.
struct DeviceBsk {
    void *bsk = nullptr;      // [n][kpl][k+1][R][NT] x 16 bytes (double2, or float4 = hi.re,hi.im,lo.re,lo.im)
    void *tables = nullptr;   // stage twiddles (stage 0 carries the twist), layout of the precision
    void *tables2 = nullptr;  // split only: the FP32 factors as broadcast pairs (build_tables_f32_paired)
    size_t bsk_bytes = 0;
    int split_shift = 0;      // split mode: weight of the high limb is 2^split_shift
};

// Device-side keyswitching key in the two layouts of the two keyswitch kernels (keyswitch.cu).
struct DeviceKsk {
    int32_t *rows = nullptr;   // per-gate kernel: [kN][t][base][stride], rows zero padded
    int stride = 0;            // padded row length (multiple of 4 >= n+1)
    int32_t *tiles = nullptr;  // tiled kernel: [slice][kN][t][base-1][tile_rs] (h = 0 rows dropped)
    int tile_cw = 0;           // output columns per warp of the tiled kernel (0: tiled kernel unavailable)
    int tile_slices = 0;       // column slices of 4 * tile_cw columns covering n+1
    int tile_slots = 0;        // resident CTAs of the tiled kernel on the device
    int32_t *rk = nullptr;     // register-key kernel: [slice][kN][t][base-1][32*rk_c]
    int rk_c = 0;              // output columns per lane of the register-key kernel (0: unavailable)
    int rk_slices = 0;         // column blocks of 32 * rk_c columns covering n+1
    int rk_slots = 0;          // resident CTAs of the register-key kernel on the device
    uint8_t *mma = nullptr;    // tensor-core kernel: [group][kN][8 KB], the B operand's shared-memory image
    int mma_groups = 0;        // 64-column groups covering n+1 (0: tensor-core kernel unavailable)
};

// What a reference parameter file carries beyond tfheb_params: the LWE and TLWE alpha_max
// (0.012467 in the reference's default sets, tfhe_gate_bootstrapping.cpp:26-75).
struct ParamMeta {
    double in_alpha_max = 0.012467;
    double tlwe_alpha_max = 0.012467;
};

// Blind-rotation variant choice of a key for one precision.  `tuned` indexes the autotuner's
// candidates of (N, l, precision).  A batch that fits one wave of CTAs with g < kSmallNeeds
// bootstraps per CTA, fewer than the tuned variant packs, runs small[g] instead: a compiled variant
// (index into the whole table, br_variant_info), -1 for the tuned one, or -2 for the default rule
// (the variant with the fewest bootstraps per CTA that still fits one wave).  tfheb_autotune fills
// small[] from one-wave timings.
constexpr int kSmallNeeds = 8;
struct BrChoice {
    int tuned = 0;
    int small[kSmallNeeds] = {-2, -2, -2, -2, -2, -2, -2, -2};
};

struct CloudKey {
    tfheb_params p{};
    ParamMeta meta;
    double ks_var = -1, bk_var = -1;  // stored key variances of a loaded file (< 0: stdev^2 on save)
    std::vector<int32_t> bsk_coef;  // [n][kpl][k+1][N] coefficient domain (host)
    std::vector<int32_t> ksk;       // [kN][t][base][n+1] (host)
    // device state
    int device = -1;
    DeviceBsk dbsk[2];              // [TFHEB_FP64], [TFHEB_SPLIT_FP32]
    DeviceKsk dksk;
    int ks_kernel = 0;              // 0 = default, 1 = per-sample, 2 = tiled, 3 = register-key, 4 = tensor-core
    cudaStream_t stream = nullptr;
    // scratch (grown on demand)
    int32_t *d_bara = nullptr;
    size_t bara_cap = 0;
    int32_t *d_acc = nullptr;
    size_t acc_cap = 0;
    int32_t *d_ksin = nullptr;
    size_t ksin_cap = 0;
    int32_t *d_io = nullptr;        // device copies of host batches: a,b,c,out
    size_t io_cap = 0;
    int32_t *d_terms = nullptr;     // keyswitch term counts of a host batch (tfheb_gate_batch_terms)
    size_t terms_cap = 0;
    cudaEvent_t scratch_done = nullptr;  // the last call using the scratch above finished with it
    BootDesc *d_bdesc = nullptr;
    size_t bdesc_cap = 0;
    GateDesc *d_gdesc = nullptr;
    size_t gdesc_cap = 0;
    int cached_gate = -1, cached_count = -1;
    int32_t *d_err = nullptr;       // device error word (bounded waits that ran out)
    uint64_t wait_timeout_ns = 1000000000ull;  // limit of every device-side wait
    int stall_producer = 0;         // test hook: the key-streaming warp issues nothing
    BrChoice br[2];                 // blind-rotation launch variants per precision
    int launches = 0;               // kernels launched (for the bench's launch count)
    // optional per-kernel timing with CUDA events on the launching stream
    bool prof = false;
    struct ProfRec {
        int which;
        cudaEvent_t a, b;
    };
    std::vector<ProfRec> prof_pending;
    double prof_ms[4] = {0, 0, 0, 0};  // prologue, blind rotation, extraction, keyswitch
    int64_t prof_n[4] = {0, 0, 0, 0};
};

struct SecretKey {
    tfheb_params p{};
    std::vector<int32_t> lwe_key;   // [n]
    std::vector<int32_t> tlwe_key;  // [k][N]
};

// ---- host helpers (host_keys.cu) ------------------------------------------------------------
void keygen(const tfheb_params &p, uint64_t seed, SecretKey &sk, CloudKey &ck);
void encrypt(const SecretKey &sk, const int32_t *bits, int32_t count, uint64_t seed, int32_t *out);
int32_t phase(const SecretKey &sk, const int32_t *ct);
void encrypt_torus(int n, const int32_t *key, const int32_t *mu, int32_t count, double stdev, uint64_t seed,
                   int32_t *out);
int32_t double_to_torus32(double d);
int32_t approx_phase(int32_t phase, int32_t msize);
int32_t modswitch_to_torus32(int32_t mu, int32_t msize);
int32_t modswitch_from_torus32(int32_t phase, int32_t msize);

// FFT-domain key preparation (host FP64), layout-compatible with the kernels.
void build_tables_fp64(int N, std::vector<double> &tables);  // complex pairs (re,im)
void build_tables_f32(int N, std::vector<float> &tables);    // float4 pairs of factors (tw4_offset)
// the same FP32 factors as {re, re, im, im} per factor, in the FP64 table's order (tw_offset)
void build_tables_f32_paired(int N, std::vector<float> &tables);
void fill_slot_freq(int N, std::vector<int32_t> &slot_freq); // [R][NT] -> frequency index
// key_transform.cu: coefficient-domain bootstrapping key [n][kpl][k+1][N] on the device -> the
// FFT-domain layout of `precision` (d_out: n*kpl*(k+1)*N/2*16 bytes), on stream s.
cudaError_t launch_bsk_to_fft(const tfheb_params &p, int precision, const int32_t *d_coef, const double *d_tables64,
                              void *d_out, int split_shift, cudaStream_t s);

// ---- kernel launchers (kernels.cu) ----------------------------------------------------------
cudaError_t launch_prologue(const tfheb_params &p, const BootDesc *d_desc, int boots, const int32_t *a,
                            const int32_t *b, const int32_t *c, int32_t *bara, int bara_stride, cudaStream_t s);
cudaError_t launch_blind_rotate(const tfheb_params &p, int precision, const DeviceBsk &bsk, const int32_t *bara,
                                int bara_stride, int boots, int nsteps, int32_t mu, const int32_t *acc_in,
                                int32_t *acc_out, cudaStream_t s, int32_t *d_err, int stall_producer,
                                uint64_t timeout_ns, const BrChoice &choice);
// The same with one compiled variant given by its index into the whole table (for timing).
cudaError_t launch_blind_rotate_exact(const tfheb_params &p, int precision, const DeviceBsk &bsk, const int32_t *bara,
                                      int bara_stride, int boots, int nsteps, int32_t mu, const int32_t *acc_in,
                                      int32_t *acc_out, cudaStream_t s, int32_t *d_err, int stall_producer,
                                      uint64_t timeout_ns, int global_index);
// Size of the whole compiled table and one entry's shape; tuned = an autotuner candidate.
int br_variant_count();
void br_variant_info(int global_index, int *N, int *l, int *precision, int *G, int *D, int *tuned);
// FFT plan of a compiled variant: 0 = one transform per thread (radix-8 team FFT), 1 = two transforms
// per thread on packed f32x2 with the digit spectra in tensor memory (split-FP32 only)
int br_variant_plan(int global_index);
// Plans of the launch variants of (N, l, precision), in the order of br_variants.
int br_variant_plans(int N, int l, int precision, int *plan, int cap);
// Index into the whole table of the `tuned`-th autotuner candidate of (N, l, precision), or -1.
int br_tuned_global(int N, int l, int precision, int tuned);
// Launch variants compiled for (N, l, precision): count, and their (G, D) into the arrays (up to cap).
int br_variants(int N, int l, int precision, int *G, int *D, int cap);
// d_desc == nullptr: row g is the plain extraction of accumulator g (no MUX term, no constant)
cudaError_t launch_extract(const tfheb_params &p, const GateDesc *d_desc, int count, const int32_t *acc,
                           int32_t *out, int out_stride, cudaStream_t s);
// acc[g] = (0, X^{2N - barb[g]} * v[g]): v [count][N], acc [count][k+1][N]
cudaError_t launch_testvec(const tfheb_params &p, int count, const int32_t *v, const int32_t *barb, int32_t *acc,
                           cudaStream_t s);
// terms[g] = number of non-zero keyswitch digits of extracted sample g (rows of in_stride int32)
cudaError_t launch_ks_terms(const tfheb_params &p, int count, const int32_t *in, int in_stride, int32_t *terms,
                            cudaStream_t s);
// out[g] = bsk_0 (x) in[g] (the first TGSW sample of `bsk`, which the caller may offset to any step):
// in/out [count][k+1][N]
cudaError_t launch_extern_product(const tfheb_params &p, int precision, const DeviceBsk &bsk, int count,
                                  const int32_t *in, int32_t *out, cudaStream_t s, int32_t *d_err,
                                  uint64_t timeout_ns);
// blind_rotate_paired.cu: the split-FP32 variants with two transforms per thread (plan 1)
struct BrArgs;
template <int N, int L, int G, int D, int XB, bool PW>
cudaError_t launch_paired(const BrArgs &a, cudaStream_t s);
// the same with a producer warp, the step's rotated words parked in TMEM during the forward
// transforms, and the first two digit pairs' forward transforms interleaved (il); also both outputs'
// inverse transforms interleaved (il2); also output 0's inverse input parked in TMEM during output
// 1's multiply-accumulate (il3); also half of each digit's keys loaded one digit ahead (il7)
template <int N, int L, int G, int D, int XB>
cudaError_t launch_paired_il(const BrArgs &a, cudaStream_t s);
template <int N, int L, int G, int D, int XB>
cudaError_t launch_paired_il2(const BrArgs &a, cudaStream_t s);
template <int N, int L, int G, int D, int XB>
cudaError_t launch_paired_il3(const BrArgs &a, cudaStream_t s);
template <int N, int L, int G, int D, int XB>
cudaError_t launch_paired_il7(const BrArgs &a, cudaStream_t s);
// keyswitch.cu: device key upload (both layouts) and the keyswitch of `count` extracted samples
// (rows of in_stride int32) into rows of n+1 int32.
cudaError_t upload_keyswitch_key(CloudKey &ck);
cudaError_t upload_keyswitch_key_mma(CloudKey &ck);  // keyswitch_mma.cu
cudaError_t launch_keyswitch_mma(const CloudKey &ck, int count, const int32_t *in, int in_stride, int32_t *out,
                                 cudaStream_t s);
void free_keyswitch_key(DeviceKsk &d);
cudaError_t launch_keyswitch(const CloudKey &ck, int count, const int32_t *in, int in_stride, int32_t *out,
                             cudaStream_t s);
int blind_rotate_supported(const tfheb_params &p);
cudaError_t launch_negate(const int32_t *in, int32_t *out, size_t count, cudaStream_t s);

int default_split_shift(const tfheb_params &p);
cudaError_t measure_fma_peak(int precision, double *tflops);

// ---- helpers shared with the allocation-free entry point (engine.cu) -------------------------
// Checks that the key is on its device with an FFT-domain key for `precision` and makes that
// device current.
tfheb_status prepare_device(CloudKey &ck, int precision);
// Linear combination of a binary gate (boot-gates.cpp:34-319): constant and operand weights.
void gate_form(int gate, int32_t *cst, int32_t *sa, int32_t *sb);
int bara_stride_for(const tfheb_params &p);
// Reads and clears the key's device error word (after the work has finished): TFHEB_ERR_TIMEOUT when
// a bounded device-side wait expired.
tfheb_status check_device_error(CloudKey &ck);
// TFHEB_ERR_INVALID (with a message) unless ptr is NULL, managed memory, or device memory on the
// key's GPU.
tfheb_status check_device_ptr(const CloudKey &ck, const void *ptr, const char *what);
extern std::atomic<int64_t> g_kernel_launches;
// Waits for the key's own stream (not the whole device) and reports a device-side wait that ran out.
tfheb_status sync_key_stream(tfheb_cloud_key *c);

// ---- reference file format (io.cu) ----------------------------------------------------------
namespace io {
bool write_params(FILE *f, const tfheb_params &p, const ParamMeta &m);
bool read_params(FILE *f, tfheb_params &p, ParamMeta &m);
bool write_cloud_content(FILE *f, const CloudKey &ck);
bool read_cloud_content(FILE *f, tfheb_params &p, CloudKey &ck);
bool write_secret_content(FILE *f, const SecretKey &sk);
bool read_secret_content(FILE *f, const tfheb_params &p, SecretKey &sk);
bool write_lwe_sample(FILE *f, int32_t n, const int32_t *a, int32_t b, double variance);
bool read_lwe_sample(FILE *f, int32_t n, int32_t *a, int32_t *b, double *variance);
}  // namespace io

// ---- errors ---------------------------------------------------------------------------------
void set_error(const std::string &msg);

}  // namespace tfheb

struct tfheb_secret_key {
    tfheb::SecretKey sk;
};
struct tfheb_cloud_key {
    tfheb::CloudKey ck;
    std::mutex mu;  // serialises host callers sharing one key (scratch buffers are per key)
};
