// key_transform.cu -- the bootstrapping key to the FFT domain on the GPU (replaces the host
// loop of init_LweBootstrappingKeyFFT / tGswToFFTConvert, lwe-bootstrapping-functions-fft.cpp:23-52).
//
// Every coefficient-domain key polynomial (n x (k+1)l x (k+1) of them) goes through the same FP64
// folded negacyclic team FFT that the blind rotation applies to its digit polynomials, so the
// spectrum comes out in the kernels' slot order with no reordering.  Each slot is scaled by 1/M
// (exact, a power of two) and stored as
//   FP64:       double2 (re, im) at [R][NT]
//   split FP32: the polynomial is first cut into limbs c = hi * 2^S + lo, lo in [-2^(S-1), 2^(S-1));
//               each limb is transformed in FP64 and rounded to float; per register pair (2m, 2m+1)
//               and limb, float4 {re(2m), re(2m+1), im(2m), im(2m+1)} at [4][2][NT]
// One team of N/16 threads per polynomial, 4 teams per CTA, twiddles in shared memory.
#include <cuda_runtime.h>
#include <stdint.h>

#include "fft.cuh"
#include "internal.h"

namespace tfheb {

namespace {

constexpr int kTeams = 4;

template <int N>
struct KtLayout {
    static constexpr int M = N / 2, NT = M / kR;
    static constexpr int TW = tw_offset<M>(FftPlan<M>::NS);
    static constexpr size_t tables_bytes = ((sizeof(cplx<double>) * TW) + 15) / 16 * 16;
    static constexpr size_t xbuf = ((size_t)Exch<double, M>::bytes + 15) / 16 * 16;
    static constexpr size_t bytes = tables_bytes + (size_t)kTeams * 2 * xbuf;
};

template <int N, bool SPLIT>
__global__ void __launch_bounds__(kTeams *(N / 16)) bsk_to_fft_kernel(const int32_t *__restrict__ coef, int polys,
                                                                     const double *__restrict__ tables,
                                                                     uint8_t *__restrict__ out, int split_shift) {
    using Lay = KtLayout<N>;
    constexpr int M = Lay::M, NT = Lay::NT;
    using F = TeamFft<double, M, kR>;
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x;
    {
        const int4 *g = reinterpret_cast<const int4 *>(tables);
        int4 *s = reinterpret_cast<int4 *>(smem);
        for (int i = tid; i < (int)(Lay::tables_bytes / 16); i += blockDim.x) s[i] = g[i];
    }
    __syncthreads();
    const int team = tid / NT, t = tid - team * NT;
    const int poly = blockIdx.x * kTeams + team;
    if (poly >= polys) return;  // a whole team; its named barrier is its own
    const int bar_id = 1 + team;
    const cplx<double> *s_tw = reinterpret_cast<const cplx<double> *>(smem);
    ExchPair xp{smem + Lay::tables_bytes + (size_t)team * 2 * Lay::xbuf, (uint32_t)Lay::xbuf, 0u};
    const int32_t *c = coef + (size_t)poly * N;
    const double scale = 1.0 / M;
    if constexpr (!SPLIT) {
        cplx<double> x[kR];
#pragma unroll
        for (int r = 0; r < kR; r++) {
            const int j = t + NT * r;
            x[r] = {(double)c[j], -(double)c[j + M]};  // a_j - i a_{j+M}; the twist is inside the FFT
        }
        F::forward(x, xp, s_tw, t, bar_id);
        double2 *o = reinterpret_cast<double2 *>(out + (size_t)poly * M * 16);
#pragma unroll
        for (int r = 0; r < kR; r++) o[r * NT + t] = make_double2(x[r].re * scale, x[r].im * scale);
    } else {
        const int64_t half = (int64_t)1 << (split_shift - 1), mask = ((int64_t)1 << split_shift) - 1;
        cplx<double> xh[kR], xl[kR];
#pragma unroll
        for (int r = 0; r < kR; r++) {
            const int j = t + NT * r;
            const int64_t v0 = c[j], v1 = c[j + M];
            const int64_t l0 = ((v0 + half) & mask) - half, l1 = ((v1 + half) & mask) - half;
            xh[r] = {(double)((v0 - l0) >> split_shift), -(double)((v1 - l1) >> split_shift)};
            xl[r] = {(double)l0, -(double)l1};
        }
        F::forward(xh, xp, s_tw, t, bar_id);
        F::forward(xl, xp, s_tw, t, bar_id);
        float4 *o = reinterpret_cast<float4 *>(out + (size_t)poly * M * 16);
#pragma unroll
        for (int m = 0; m < kR / 2; m++) {
            o[(m * 2 + 0) * NT + t] = make_float4((float)(xh[2 * m].re * scale), (float)(xh[2 * m + 1].re * scale),
                                                  (float)(xh[2 * m].im * scale), (float)(xh[2 * m + 1].im * scale));
            o[(m * 2 + 1) * NT + t] = make_float4((float)(xl[2 * m].re * scale), (float)(xl[2 * m + 1].re * scale),
                                                  (float)(xl[2 * m].im * scale), (float)(xl[2 * m + 1].im * scale));
        }
    }
}

template <int N, bool SPLIT>
cudaError_t launch_n(const int32_t *coef, int polys, const double *tables, void *out, int split_shift,
                     cudaStream_t s) {
    using Lay = KtLayout<N>;
    auto kern = bsk_to_fft_kernel<N, SPLIT>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::bytes);
    if (e != cudaSuccess) return e;
    const int grid = (polys + kTeams - 1) / kTeams;
    kern<<<grid, kTeams * Lay::NT, Lay::bytes, s>>>(coef, polys, tables, static_cast<uint8_t *>(out), split_shift);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_bsk_to_fft(const tfheb_params &p, int precision, const int32_t *d_coef, const double *d_tables64,
                              void *d_out, int split_shift, cudaStream_t s) {
    const int polys = p.n * (p.k + 1) * p.l * (p.k + 1);
    const bool split = precision == TFHEB_SPLIT_FP32;
    switch (p.N) {
        case 512: return split ? launch_n<512, true>(d_coef, polys, d_tables64, d_out, split_shift, s)
                               : launch_n<512, false>(d_coef, polys, d_tables64, d_out, split_shift, s);
        case 1024: return split ? launch_n<1024, true>(d_coef, polys, d_tables64, d_out, split_shift, s)
                                : launch_n<1024, false>(d_coef, polys, d_tables64, d_out, split_shift, s);
        case 2048: return split ? launch_n<2048, true>(d_coef, polys, d_tables64, d_out, split_shift, s)
                                : launch_n<2048, false>(d_coef, polys, d_tables64, d_out, split_shift, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace tfheb
