// dft_probe.cu -- measures whether a radix-8 stage of the blind rotation's FFT would run faster on
// the tensor cores than on the CUDA cores (the decision the FFT design rests on).
//
// Three ways to apply 8-point complex DFTs to register-resident data, each repeated many times per
// thread with the result fed back as the next input (scaled by 1/8, exact, so values stay bounded):
//   0  CUDA cores: the FFT's own dft8 codelet (fft.cuh), one 8-point column per thread;
//   1  tensor cores, compute only: the DFT as a real 16x16 matrix [[Fr, -Fi], [Fi, Fr]] times a
//      16 x 8 block of columns (re parts, then im parts), with mma.sync m16n8k8 TF32 in three passes
//      (A_hi B_hi + A_hi B_lo + A_lo B_hi, FP32 accumulation) to reach FP32 accuracy; the output is
//      re-split and fed back in the accumulator's own lane layout (an idealised upper bound that no
//      FFT can use as is, because an FFT needs the outputs as the next stage's inputs);
//   2  tensor cores as an FFT would use them: as 1, plus moving each output block from the
//      accumulator layout into the input-operand layout with warp shuffles, as the next stage needs.
// Reported: device time per 8-point DFT over the whole GPU, and the largest error relative to the
// column's norm against FP64 DFTs of the same inputs (host side).
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>
#include <complex>
#include <vector>

#include "fft.cuh"
#include "internal.h"

namespace tfheb {
namespace {

constexpr int kProbeIters = 2048;

__global__ void dft8_core_kernel(float2 *data, int iters) {
    const size_t col = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    cplx<float> x[8];
#pragma unroll
    for (int r = 0; r < 8; r++) {
        const float2 v = data[col * 8 + r];
        x[r] = {v.x, v.y};
    }
    for (int it = 0; it < iters; it++) {
        dft8<float, false>(x);
#pragma unroll
        for (int r = 0; r < 8; r++) x[r] = {x[r].re * 0.125f, x[r].im * 0.125f};
    }
#pragma unroll
    for (int r = 0; r < 8; r++) data[col * 8 + r] = make_float2(x[r].re, x[r].im);
}

// TF32 hi / lo split of a float (hi rounded to TF32, lo the exact remainder rounded to TF32)
__device__ __forceinline__ void split_tf32(float v, uint32_t &hi, uint32_t &lo) {
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(hi) : "f"(v));
    const float rest = v - __uint_as_float(hi);
    asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(lo) : "f"(rest));
}

__device__ __forceinline__ void mma_tf32(float (&d)[4], const uint32_t (&a)[4], uint32_t b0, uint32_t b1) {
    asm volatile(
        "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0, %1, %2, %3}, {%4, %5, %6, %7}, {%8, %9}, "
        "{%0, %1, %2, %3};"
        : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// Real DFT matrix element (row i < 16: output re (i < 8) / im; col j < 16: input re (j < 8) / im).
__device__ __forceinline__ double dft_real(int i, int j) {
    const int k = i & 7, n = j & 7;
    const double ang = -2.0 * 3.14159265358979323846 * (double)(k * n) / 8.0;
    const double fr = cos(ang), fi = sin(ang);
    if (i < 8) return j < 8 ? fr : -fi;  // Yr = Fr Xr - Fi Xi
    return j < 8 ? fi : fr;              // Yi = Fi Xr + Fr Xi
}

// One warp holds 8 columns: B fragments (k-step 0: re rows 0..7, k-step 1: im rows 8..15);
// thread g = lane / 4, q = lane % 4 holds rows q and q + 4 of column g of each k-step.
template <bool RELAYOUT>
__global__ void dft8_mma_kernel(float2 *data, int iters) {
    const int lane = threadIdx.x & 31, g = lane >> 2, q = lane & 3;
    const size_t block = ((size_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;  // 8 columns per warp
    const float2 *cols = data + block * 64;
    // A fragments of both k-steps, hi and lo: rows g, g+8; cols q, q+4 of the 16 x 8 slice
    uint32_t ahi[2][4], alo[2][4];
#pragma unroll
    for (int ks = 0; ks < 2; ks++) {
        const int rr[4] = {g, g + 8, g, g + 8}, cc[4] = {q, q, q + 4, q + 4};
#pragma unroll
        for (int e = 0; e < 4; e++) split_tf32((float)dft_real(rr[e], ks * 8 + cc[e]), ahi[ks][e], alo[ks][e]);
    }
    // this thread's inputs: column g, rows q and q + 4 of the re (ks 0) and im (ks 1) parts
    float b[2][2];
    b[0][0] = cols[g * 8 + q].x;
    b[0][1] = cols[g * 8 + q + 4].x;
    b[1][0] = cols[g * 8 + q].y;
    b[1][1] = cols[g * 8 + q + 4].y;
    float d[4];
    for (int it = 0; it < iters; it++) {
        d[0] = d[1] = d[2] = d[3] = 0.f;
#pragma unroll
        for (int ks = 0; ks < 2; ks++) {
            uint32_t bh0, bl0, bh1, bl1;
            split_tf32(b[ks][0], bh0, bl0);
            split_tf32(b[ks][1], bh1, bl1);
            mma_tf32(d, ahi[ks], bh0, bh1);
            mma_tf32(d, ahi[ks], bl0, bl1);
            mma_tf32(d, alo[ks], bh0, bh1);
        }
        // d: rows g (re of output g) and g + 8 (im), columns 2q, 2q+1
        if constexpr (RELAYOUT) {
            // next input: column g, rows q and q + 4 = output rows held by lane (row * 4 + g / 2)
            const int src0 = q * 4 + (g >> 1), src1 = (q + 4) * 4 + (g >> 1);
            const float r00 = __shfl_sync(0xffffffffu, d[0], src0), r01 = __shfl_sync(0xffffffffu, d[1], src0);
            const float r10 = __shfl_sync(0xffffffffu, d[0], src1), r11 = __shfl_sync(0xffffffffu, d[1], src1);
            const float i00 = __shfl_sync(0xffffffffu, d[2], src0), i01 = __shfl_sync(0xffffffffu, d[3], src0);
            const float i10 = __shfl_sync(0xffffffffu, d[2], src1), i11 = __shfl_sync(0xffffffffu, d[3], src1);
            const bool odd = g & 1;
            b[0][0] = (odd ? r01 : r00) * 0.125f;
            b[0][1] = (odd ? r11 : r10) * 0.125f;
            b[1][0] = (odd ? i01 : i00) * 0.125f;
            b[1][1] = (odd ? i11 : i10) * 0.125f;
        } else {
            b[0][0] = d[0] * 0.125f;
            b[0][1] = d[1] * 0.125f;
            b[1][0] = d[2] * 0.125f;
            b[1][1] = d[3] * 0.125f;
        }
    }
    if constexpr (RELAYOUT) {
        float2 *out = data + block * 64;
        out[g * 8 + q] = make_float2(b[0][0], b[1][0]);
        out[g * 8 + q + 4] = make_float2(b[0][1], b[1][1]);
    } else {
        // one DFT in the accumulator's layout: write it as a column block for the accuracy check
        float2 *out = data + block * 64;
        out[(2 * q) * 8 + g] = make_float2(d[0], d[2]);
        out[(2 * q + 1) * 8 + g] = make_float2(d[1], d[3]);
    }
}

}  // namespace

cudaError_t measure_dft8(int method, double *ns_per_dft, double *max_rel_err) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int threads = 256, blocks = sms * 8;
    const size_t nthreads = (size_t)threads * blocks;
    const size_t cols = method == 0 ? nthreads : nthreads / 32 * 8;  // 8-point columns in flight
    std::vector<float2> h(cols * 8);
    uint64_t s = 0x12345678ull;
    for (auto &v : h) {
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        const float a = (float)((double)(s >> 40) / (double)(1ull << 24) - 0.5);
        s = s * 6364136223846793005ull + 1442695040888963407ull;
        const float bb = (float)((double)(s >> 40) / (double)(1ull << 24) - 0.5);
        v = make_float2(a, bb);
    }
    float2 *d = nullptr;
    cudaError_t e = cudaMalloc(&d, h.size() * sizeof(float2));
    if (e != cudaSuccess) return e;
    auto launch = [&](int iters) {
        if (method == 0) dft8_core_kernel<<<blocks, threads>>>(d, iters);
        else if (method == 1) dft8_mma_kernel<false><<<blocks, threads>>>(d, iters);
        else dft8_mma_kernel<true><<<blocks, threads>>>(d, iters);
    };
    // accuracy: one application against an FP64 DFT (the exact 1/8 scaling is undone)
    cudaMemcpy(d, h.data(), h.size() * sizeof(float2), cudaMemcpyHostToDevice);
    launch(1);
    std::vector<float2> out(h.size());
    cudaMemcpy(out.data(), d, out.size() * sizeof(float2), cudaMemcpyDeviceToHost);
    double worst = 0;
    const size_t check = std::min<size_t>(cols, 4096);
    for (size_t c = 0; c < check; c++) {
        double norm = 0;
        for (int n = 0; n < 8; n++) norm += (double)h[c * 8 + n].x * h[c * 8 + n].x + (double)h[c * 8 + n].y * h[c * 8 + n].y;
        norm = std::sqrt(norm);
        for (int k = 0; k < 8; k++) {
            std::complex<double> y = 0;
            for (int n = 0; n < 8; n++)
                y += std::complex<double>(h[c * 8 + n].x, h[c * 8 + n].y) * std::polar(1.0, -2.0 * M_PI * k * n / 8.0);
            // method 0 keeps outputs in the codelet's natural order, scaled by 1/8 (exact)
            const double scale = method == 1 ? 1.0 : 0.125;
            const std::complex<double> got(out[c * 8 + k].x / scale, out[c * 8 + k].y / scale);
            worst = std::max(worst, std::abs(got - y) / std::max(norm, 1e-30));
        }
    }
    *max_rel_err = worst;
    // throughput
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0);
        launch(kProbeIters);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) best = std::min(best, ms);
    }
    e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    *ns_per_dft = (double)best * 1e6 / ((double)cols * kProbeIters);
    return e;
}

}  // namespace tfheb

extern "C" tfheb_status tfheb_measure_dft8(int32_t device, int32_t method, double *ns_per_dft, double *max_rel_err) {
    if (!ns_per_dft || !max_rel_err || method < 0 || method > 2) return TFHEB_ERR_INVALID;
    if (cudaSetDevice(device) != cudaSuccess) {
        tfheb::set_error("tfheb_measure_dft8: no such device");
        return TFHEB_ERR_NO_DEVICE;
    }
    const cudaError_t e = tfheb::measure_dft8(method, ns_per_dft, max_rel_err);
    if (e != cudaSuccess) {
        tfheb::set_error(std::string("tfheb_measure_dft8: ") + cudaGetErrorString(e));
        return TFHEB_ERR_CUDA;
    }
    return TFHEB_OK;
}
