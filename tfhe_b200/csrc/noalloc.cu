// noalloc.cu -- the batched gate pipeline for callers that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not available or not allowed -- a real-time or
// signal-handling context that must not take the allocator's locks or block on it, or a host
// process whose device memory is carved up by a framework that forbids allocations outside its own
// pool.  tfheb_gate_batch_device grows per-key scratch buffers with cudaMalloc on demand; this
// variant instead takes all of its scratch from one file-scope device array, so a call allocates
// nothing.
//
// Scratch: g_noalloc_scratch, kNoAllocScratchBytes = 8 MiB, held by every GPU that loads the library
// until the process exits.  One call needs, per gate (MUX: two bootstraps per gate),
//     bootstraps * (12 + 4*((n+4)&~3) + 4*(k+1)*N) + gates * (12 + 4*(k*N+1)) bytes
// (plus 256-byte alignment of each region); the default 128-bit parameters fit 565 binary gates or
// 327 MUX gates per call, the N=2048 set 301 binary or 176 MUX gates.  Larger batches are rejected
// with TFHEB_ERR_INVALID; split them into several calls.
//
// Set-up: the first call on a device looks up the array's device address (cudaGetSymbolAddress,
// with that device current) and caches it; make that first call before any stream capture.  The
// cached address belongs to the device's context: a process that calls cudaDeviceReset must not
// call this entry point on that device afterwards.
//
// The array is shared by every call in the process on that device and keeps the previous call's
// contents.  Nothing in it has to start at zero: the descriptors are rewritten by a kernel at the
// start of each call and every other region is fully written before it is read.  Calls whose work
// overlaps on the GPU (different streams, or different threads without ordering) race on the array;
// serialise them on one stream.
#include <cuda_runtime.h>

#include <mutex>

#include "internal.h"

namespace tfheb {
namespace {

constexpr size_t kNoAllocScratchBytes = size_t(8) << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_ptr_mu;
void *g_scratch_ptr[kMaxDevices] = {};

// Device address of the scratch array on the current device.  In host code g_noalloc_scratch is
// only a stand-in symbol, so the address is looked up once per device, with that device current.
cudaError_t scratch_address(int device, void **ptr) {
    if (device < 0 || device >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_ptr_mu);
    if (!g_scratch_ptr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        g_scratch_ptr[device] = p;
    }
    *ptr = g_scratch_ptr[device];
    return cudaSuccess;
}

size_t align256(size_t x) { return (x + 255) & ~size_t(255); }

// Descriptors of a uniform batch, written on the device (no host copy).
__global__ void fill_descs_kernel(BootDesc *bd, GateDesc *gd, int count, int mux, int32_t cst, int sa, int sb,
                                  int32_t and_c, int32_t mu8) {
    const int g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= count) return;
    if (mux) {  // boot-gates.cpp:329-370: (0,-1/8)+a+b and (0,-1/8)-a+c, then + (0,1/8)
        bd[2 * g] = BootDesc{g, and_c, 1, 1, 0, 1};
        bd[2 * g + 1] = BootDesc{g, and_c, -1, 1, 0, 2};
        gd[g] = GateDesc{2 * g, 2 * g + 1, mu8};
    } else {
        bd[g] = BootDesc{g, cst, (int8_t)sa, (int8_t)sb, 0, 1};
        gd[g] = GateDesc{g, -1, 0};
    }
}

}  // namespace
}  // namespace tfheb

using namespace tfheb;

extern "C" tfheb_status tfheb_gate_batch_device_noalloc(tfheb_cloud_key *c, int32_t gate, int32_t precision,
                                                        int32_t count, const int32_t *d_a, const int32_t *d_b,
                                                        const int32_t *d_c, int32_t *d_out, void *stream) {
    if (!c || count < 0 || gate < 0 || gate > TFHEB_COPY) return TFHEB_ERR_INVALID;
    if (count > 0 && (!d_a || !d_out || (gate == TFHEB_MUX && (!d_b || !d_c)) || (gate < TFHEB_MUX && !d_b)))
        return TFHEB_ERR_INVALID;
    // far above what the fixed array holds at any parameter set; keeps the size arithmetic in range
    constexpr int32_t kMaxCount = 1 << 20;
    if (count > kMaxCount) {
        set_error("tfheb_gate_batch_device_noalloc: " + std::to_string(count) +
                  " gates exceed the fixed scratch array by far; split the batch");
        return TFHEB_ERR_INVALID;
    }
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    tfheb_status st = prepare_device(ck, precision);
    if (st != TFHEB_OK) return st;
    if (count == 0) return TFHEB_OK;
    // a host pointer or another GPU's memory would fault inside the kernels instead of returning
    // an error (cudaPointerGetAttributes allocates nothing)
    const void *bufs[4] = {d_a, d_b, d_c, d_out};
    const char *names[4] = {"d_a", "d_b", "d_c", "d_out"};
    for (int i = 0; i < 4; i++)
        if ((st = check_device_ptr(ck, bufs[i], names[i])) != TFHEB_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : ck.stream;
    const tfheb_params &p = ck.p;
    const int n1 = p.n + 1;
    if (gate == TFHEB_COPY || gate == TFHEB_NOT) {  // bootstrap-free: no scratch needed
        cudaError_t e = gate == TFHEB_COPY
                            ? cudaMemcpyAsync(d_out, d_a, (size_t)count * n1 * 4, cudaMemcpyDeviceToDevice, s)
                            : launch_negate(d_a, d_out, (size_t)count * n1, s);
        if (e != cudaSuccess) {
            set_error(std::string("tfheb_gate_batch_device_noalloc: ") + cudaGetErrorString(e));
            return TFHEB_ERR_CUDA;
        }
        if (gate == TFHEB_NOT) g_kernel_launches += 1;
        return TFHEB_OK;
    }
    const size_t boots = gate == TFHEB_MUX ? 2 * (size_t)count : (size_t)count;
    const size_t bs = (size_t)bara_stride_for(p);
    const size_t kN1 = (size_t)p.k * p.N + 1;
    const size_t off_bd = 0;
    const size_t off_gd = off_bd + align256(sizeof(BootDesc) * boots);
    const size_t off_bara = off_gd + align256(sizeof(GateDesc) * (size_t)count);
    const size_t off_acc = off_bara + align256(4 * boots * bs);
    const size_t off_ksin = off_acc + align256(4 * boots * (p.k + 1) * (size_t)p.N);
    const size_t need = off_ksin + align256(4 * (size_t)count * kN1);
    if (need > kNoAllocScratchBytes) {
        set_error("tfheb_gate_batch_device_noalloc: " + std::to_string(count) + " gates need " +
                  std::to_string(need) + " bytes of scratch, more than the fixed " +
                  std::to_string(kNoAllocScratchBytes) + "-byte device array; split the batch");
        return TFHEB_ERR_INVALID;
    }
    void *base = nullptr;
    cudaError_t e = scratch_address(ck.device, &base);
    if (e != cudaSuccess) {
        set_error(std::string("tfheb_gate_batch_device_noalloc: cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        return TFHEB_ERR_CUDA;
    }
    unsigned char *b = static_cast<unsigned char *>(base);
    BootDesc *bd = reinterpret_cast<BootDesc *>(b + off_bd);
    GateDesc *gd = reinterpret_cast<GateDesc *>(b + off_gd);
    int32_t *bara = reinterpret_cast<int32_t *>(b + off_bara);
    int32_t *acc = reinterpret_cast<int32_t *>(b + off_acc);
    int32_t *ksin = reinterpret_cast<int32_t *>(b + off_ksin);

    int32_t cst = 0, sa = 0, sb = 0;
    if (gate != TFHEB_MUX) gate_form(gate, &cst, &sa, &sb);
    fill_descs_kernel<<<(count + 255) / 256, 256, 0, s>>>(bd, gd, count, gate == TFHEB_MUX, cst, sa, sb,
                                                        modswitch_to_torus32(-1, 8), modswitch_to_torus32(1, 8));
    if ((e = cudaGetLastError()) == cudaSuccess)
        e = launch_prologue(p, bd, (int)boots, d_a, d_b, d_c, bara, (int)bs, s);
    if (e == cudaSuccess)
        e = launch_blind_rotate(p, precision, ck.dbsk[precision], bara, (int)bs, (int)boots, p.n,
                                modswitch_to_torus32(1, 8), nullptr, acc, s, ck.d_err, ck.stall_producer,
                                ck.wait_timeout_ns, ck.br[precision]);
    if (e == cudaSuccess) e = launch_extract(p, gd, count, acc, ksin, (int)kN1, s);
    if (e == cudaSuccess) e = launch_keyswitch(ck, count, ksin, (int)kN1, d_out, s);
    if (e != cudaSuccess) {
        set_error(std::string("tfheb_gate_batch_device_noalloc: ") + cudaGetErrorString(e));
        return TFHEB_ERR_CUDA;
    }
    g_kernel_launches += 5;
    return TFHEB_OK;
}
