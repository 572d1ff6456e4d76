// kernels.cu -- the gate-bootstrapping hot path on sm_100a.
//
//   prologue_kernel      gate linear combination + modulus switch to Z_2N   (boot-gates.cpp:34-370,
//                        lwe-bootstrapping-functions-fft.cpp:184-188, numeric-functions.cpp:59-65)
//   blind_rotate_kernel  persistent blind rotation: accumulator resident in shared memory for all
//                        n CMUX steps; per step rotation, gadget decomposition, negacyclic FFT,
//                        FFT-domain MAC against the bootstrapping key, inverse FFT, accumulate
//                        (lwe-bootstrapping-functions-fft.cpp:67-156, tgsw-fft-operations.cpp:89-114,
//                        tgsw-functions.cpp:297-410, tlwe-functions.cpp:202-206)
//   extract_kernel       sample extraction at index 0, MUX recombination   (lwe.cpp:41-60,
//                        boot-gates.cpp:360-364)
//   keyswitch_kernel     integer gather-accumulate keyswitch               (lwe-keyswitch-functions.cpp:114-238)
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>

#include "fft.cuh"
#include "internal.h"

namespace tfheb {

// ============================================================================================
// prologue
// ============================================================================================

__device__ __forceinline__ int32_t modswitch_from_dev(uint32_t phase, uint64_t interv) {
    const uint64_t phase64 = ((uint64_t)phase << 32) + (interv >> 1);
    return (int32_t)(phase64 / interv);
}

// one CTA per bootstrap, threads over the n+1 coefficients
__global__ void prologue_kernel(const BootDesc *__restrict__ desc, const int32_t *__restrict__ a,
                                const int32_t *__restrict__ b, const int32_t *__restrict__ c, int n,
                                uint64_t interv, int32_t *__restrict__ bara, int bara_stride) {
    const BootDesc d = desc[blockIdx.x];
    const int32_t *src[3] = {a, b, c};
    const uint32_t *x = reinterpret_cast<const uint32_t *>(src[d.xsel]) + (size_t)d.gate * (n + 1);
    const uint32_t *y = reinterpret_cast<const uint32_t *>(src[d.ysel]) + (size_t)d.gate * (n + 1);
    int32_t *out = bara + (size_t)blockIdx.x * bara_stride;
    for (int i = threadIdx.x; i <= n; i += blockDim.x) {
        uint32_t v = (uint32_t)(int32_t)d.sa * x[i];
        if (d.sb) v += (uint32_t)(int32_t)d.sb * y[i];
        if (i == n) v += (uint32_t)d.cst;
        out[i] = modswitch_from_dev(v, interv);
    }
}

cudaError_t launch_prologue(const tfheb_params &p, const BootDesc *d_desc, int boots, const int32_t *a,
                            const int32_t *b, const int32_t *c, int32_t *bara, int bara_stride, cudaStream_t s) {
    if (boots <= 0) return cudaSuccess;
    const uint64_t interv = ((UINT64_C(1) << 63) / (uint64_t)(2 * p.N)) * 2;
    prologue_kernel<<<boots, 256, 0, s>>>(d_desc, a, b ? b : a, c ? c : a, p.n, interv, bara, bara_stride);
    return cudaGetLastError();
}

// ============================================================================================
// blind rotation
// ============================================================================================

// Shared-memory plan of one CTA (GPB teams, one bootstrap per team).
template <typename T, int N, int K>
struct BrSmem {
    static constexpr int M = N / 2;
    static constexpr int NT = M / kR;
    static constexpr int TW = tw_offset<M>(FftPlan<M>::NS);         // stage twiddles
    static constexpr size_t tables_bytes = sizeof(cplx<T>) * (TW + kR * NT);
    static constexpr size_t team_acc = sizeof(int32_t) * (K + 1) * N;
    static constexpr size_t team_buf = 2 * sizeof(T) * M;
    __host__ __device__ static size_t team_bytes(int n) { return team_acc + team_buf + sizeof(int32_t) * ((n + 4) & ~3); }
    __host__ __device__ static size_t bytes(int gpb, int n) { return tables_bytes + gpb * team_bytes(n); }
};

// (X^a - 1) * acc, coefficient j (toruspolynomial-functions.cpp:117-136), 0 <= a < 2N
template <int N>
__device__ __forceinline__ uint32_t rot_minus_one(const uint32_t *poly, int j, int a) {
    int src = j - a;
    uint32_t v;
    if (src >= 0) v = poly[src];
    else if (src >= -N) v = 0u - poly[src + N];
    else v = poly[src + 2 * N];
    return v - poly[j];
}

template <typename T>
__device__ __forceinline__ int64_t round_to_i64(T v);
template <>
__device__ __forceinline__ int64_t round_to_i64<double>(double v) { return __double2ll_rn(v); }
template <>
__device__ __forceinline__ int64_t round_to_i64<float>(float v) { return __float2ll_rn(v); }

// Bootstrapping-key slot loads (16 bytes per slot).
template <typename T, bool SPLIT>
struct BskSlot;
template <>
struct BskSlot<double, false> {
    cplx<double> v;
    __device__ __forceinline__ void load(const void *base, size_t idx) {
        const double2 d = __ldg(reinterpret_cast<const double2 *>(base) + idx);
        v = {d.x, d.y};
    }
};
template <>
struct BskSlot<float, true> {
    cplx<float> hi, lo;
    __device__ __forceinline__ void load(const void *base, size_t idx) {
        const float4 d = __ldg(reinterpret_cast<const float4 *>(base) + idx);
        hi = {d.x, d.y};
        lo = {d.z, d.w};
    }
};

template <typename T, int N, int K, int L, bool SPLIT, int GPB>
__global__ void __launch_bounds__(GPB *(N / 2 / kR))
    blind_rotate_kernel(const int32_t *__restrict__ bara, int bara_stride, const void *__restrict__ bsk,
                        const cplx<T> *__restrict__ tables, const int32_t *__restrict__ acc_in,
                        int32_t *__restrict__ acc_out, int boots, int nsteps, int32_t mu, int Bgbit,
                        int split_shift) {
    constexpr int M = N / 2, NT = M / kR, KP1 = K + 1, KPL = KP1 * L;
    using Sm = BrSmem<T, N, K>;
    using F = TeamFft<T, M, kR>;
    extern __shared__ __align__(16) unsigned char smem[];

    // ---- CTA-wide: tables to shared memory ------------------------------------------------
    cplx<T> *s_tables = reinterpret_cast<cplx<T> *>(smem);
    for (int i = threadIdx.x; i < Sm::TW + kR * NT; i += blockDim.x) s_tables[i] = tables[i];
    __syncthreads();
    const cplx<T> *s_tw = s_tables;
    const cplx<T> *s_twist = s_tables + Sm::TW;

    const int team = threadIdx.x / NT;
    const int t = threadIdx.x - team * NT;
    const int boot = blockIdx.x * GPB + team;
    if (boot >= boots) return;  // whole team leaves; no CTA-wide barrier follows
    const int bar_id = 1 + team;

    unsigned char *tb = smem + Sm::tables_bytes + (size_t)team * Sm::team_bytes(nsteps);
    uint32_t *s_acc = reinterpret_cast<uint32_t *>(tb);
    T *buf_re = reinterpret_cast<T *>(tb + Sm::team_acc);
    T *buf_im = buf_re + M;
    int32_t *s_bara = reinterpret_cast<int32_t *>(tb + Sm::team_acc + Sm::team_buf);

    // ---- team init: bara row, accumulator ------------------------------------------------
    const int32_t *my_bara = bara + (size_t)boot * bara_stride;
    for (int i = t; i < nsteps; i += NT) s_bara[i] = my_bara[i];
    if (acc_in) {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(acc_in) + (size_t)boot * KP1 * N;
        for (int i = t; i < KP1 * N; i += NT) s_acc[i] = src[i];
    } else {
        // acc = (0, X^{2N-barb} * [mu,...,mu])  (lwe-bootstrapping-functions-fft.cpp:142-145)
        const int barb = my_bara[nsteps];
        const int e = 2 * N - barb;
        for (int i = t; i < K * N; i += NT) s_acc[i] = 0u;
        for (int j = t; j < N; j += NT) {
            int src = j - e;
            uint32_t neg = 0;
            while (src < 0) {
                src += N;
                neg ^= 1u;
            }
            s_acc[K * N + j] = neg ? 0u - (uint32_t)mu : (uint32_t)mu;
        }
    }
    team_sync(bar_id, NT);

    // gadget constants (tgsw.cpp:7-29)
    uint32_t offset = 0;
#pragma unroll
    for (int q = 0; q < L; q++) offset += 1u << (32 - (q + 1) * Bgbit);
    offset *= 1u << (Bgbit - 1);
    const uint32_t maskBg = (1u << Bgbit) - 1u;
    const int32_t halfBg = 1 << (Bgbit - 1);

    cplx<T> twist[kR];
#pragma unroll
    for (int r = 0; r < kR; r++) twist[r] = s_twist[r * NT + t];

    for (int step = 0; step < nsteps; step++) {
        const int ai = s_bara[step] & (2 * N - 1);  // rotations live in Z_2N; keeps indices in bounds
        cplx<T> acc_hi[KP1][kR];
        cplx<T> acc_lo[SPLIT ? KP1 : 1][kR];
#pragma unroll
        for (int v = 0; v < KP1; v++)
#pragma unroll
            for (int r = 0; r < kR; r++) {
                acc_hi[v][r] = {T(0), T(0)};
                if (SPLIT) acc_lo[SPLIT ? v : 0][r] = {T(0), T(0)};
            }

        const size_t bsk_step = (size_t)step * KPL * KP1 * kR * NT;
#pragma unroll 1
        for (int u = 0; u < KP1; u++) {
            const uint32_t *poly = s_acc + u * N;
            uint32_t x0[kR], x1[kR];
#pragma unroll
            for (int r = 0; r < kR; r++) {
                const int j = t + NT * r;
                x0[r] = rot_minus_one<N>(poly, j, ai) + offset;
                x1[r] = rot_minus_one<N>(poly, j + M, ai) + offset;
            }
#pragma unroll 1
            for (int q = 0; q < L; q++) {
                const int shift = 32 - (q + 1) * Bgbit;
                cplx<T> z[kR];
#pragma unroll
                for (int r = 0; r < kR; r++) {
                    const int32_t d0 = (int32_t)((x0[r] >> shift) & maskBg) - halfBg;
                    const int32_t d1 = (int32_t)((x1[r] >> shift) & maskBg) - halfBg;
                    // (a_j - i a_{j+M}) * exp(-i pi j / N)
                    z[r] = cmul(cplx<T>{T(d0), T(-d1)}, twist[r]);
                }
                F::forward(z, buf_re, buf_im, s_tw, t, bar_id);
                const int p = u * L + q;
#pragma unroll
                for (int v = 0; v < KP1; v++) {
                    const size_t base = bsk_step + ((size_t)p * KP1 + v) * kR * NT + t;
#pragma unroll
                    for (int r = 0; r < kR; r++) {
                        BskSlot<T, SPLIT> s;
                        s.load(bsk, base + (size_t)r * NT);
                        if constexpr (SPLIT) {
                            cmac(acc_hi[v][r], z[r], s.hi);
                            cmac(acc_lo[v][r], z[r], s.lo);
                        } else {
                            cmac(acc_hi[v][r], z[r], s.v);
                        }
                    }
                }
            }
        }

        // inverse transforms and accumulate (the key was pre-scaled by 1/M)
#pragma unroll
        for (int v = 0; v < KP1; v++) {
            uint32_t c0[kR], c1[kR];
            {
                cplx<T> z[kR];
#pragma unroll
                for (int r = 0; r < kR; r++) z[r] = acc_hi[v][r];
                F::inverse(z, buf_re, buf_im, s_tw, t, bar_id);
#pragma unroll
                for (int r = 0; r < kR; r++) {
                    const cplx<T> w = cmulconj(z[r], twist[r]);  // (c_j - i c_{j+M})
                    const uint64_t lo0 = (uint64_t)round_to_i64<T>(w.re);
                    const uint64_t lo1 = (uint64_t)round_to_i64<T>(-w.im);
                    if constexpr (SPLIT) {
                        c0[r] = (uint32_t)lo0 << split_shift;
                        c1[r] = (uint32_t)lo1 << split_shift;
                    } else {
                        c0[r] = (uint32_t)lo0;
                        c1[r] = (uint32_t)lo1;
                    }
                }
            }
            if constexpr (SPLIT) {
                cplx<T> z[kR];
#pragma unroll
                for (int r = 0; r < kR; r++) z[r] = acc_lo[v][r];
                F::inverse(z, buf_re, buf_im, s_tw, t, bar_id);
#pragma unroll
                for (int r = 0; r < kR; r++) {
                    const cplx<T> w = cmulconj(z[r], twist[r]);
                    c0[r] += (uint32_t)(uint64_t)round_to_i64<T>(w.re);
                    c1[r] += (uint32_t)(uint64_t)round_to_i64<T>(-w.im);
                }
            }
            uint32_t *poly = s_acc + v * N;
#pragma unroll
            for (int r = 0; r < kR; r++) {
                const int j = t + NT * r;
                poly[j] += c0[r];
                poly[j + M] += c1[r];
            }
        }
        team_sync(bar_id, NT);
    }

    uint32_t *dst = reinterpret_cast<uint32_t *>(acc_out) + (size_t)boot * KP1 * N;
    for (int i = t; i < KP1 * N; i += NT) dst[i] = s_acc[i];
}

template <typename T, int N, int K, int L, bool SPLIT, int GPB>
static cudaError_t launch_br_t(const DeviceBsk &bsk, const int32_t *bara, int bara_stride, int boots, int nsteps,
                               int32_t mu, const int32_t *acc_in, int32_t *acc_out, int Bgbit, cudaStream_t s) {
    constexpr int NT = N / 2 / kR;
    const size_t smem = BrSmem<T, N, K>::bytes(GPB, nsteps);
    auto kern = blind_rotate_kernel<T, N, K, L, SPLIT, GPB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = (boots + GPB - 1) / GPB;
    kern<<<grid, GPB * NT, smem, s>>>(bara, bara_stride, bsk.bsk, reinterpret_cast<const cplx<T> *>(bsk.tables),
                                      acc_in, acc_out, boots, nsteps, mu, Bgbit, bsk.split_shift);
    return cudaGetLastError();
}

int blind_rotate_supported(const tfheb_params &p) {
    // teams of N/16 threads synchronise with named barriers, which need whole warps: N >= 512
    if (p.k != 1 || p.l != 3) return 0;
    return p.N == 512 || p.N == 1024 || p.N == 2048;
}

template <int N>
static cudaError_t launch_br_n(int precision, const DeviceBsk &bsk, const int32_t *bara, int bara_stride,
                               int boots, int nsteps, int32_t mu, const int32_t *acc_in, int32_t *acc_out, int Bgbit,
                               cudaStream_t s, int gpb) {
    if (precision == TFHEB_FP64) {
        if (gpb >= 2)
            return launch_br_t<double, N, 1, 3, false, 2>(bsk, bara, bara_stride, boots, nsteps, mu, acc_in, acc_out,
                                                         Bgbit, s);
        return launch_br_t<double, N, 1, 3, false, 1>(bsk, bara, bara_stride, boots, nsteps, mu, acc_in, acc_out,
                                                     Bgbit, s);
    }
    if (gpb >= 2)
        return launch_br_t<float, N, 1, 3, true, 2>(bsk, bara, bara_stride, boots, nsteps, mu, acc_in, acc_out, Bgbit,
                                                   s);
    return launch_br_t<float, N, 1, 3, true, 1>(bsk, bara, bara_stride, boots, nsteps, mu, acc_in, acc_out, Bgbit, s);
}

cudaError_t launch_blind_rotate(const tfheb_params &p, int precision, const DeviceBsk &bsk, const int32_t *bara,
                                int bara_stride, int boots, int nsteps, int32_t mu, const int32_t *acc_in,
                                int32_t *acc_out, cudaStream_t s, int gpb) {
    if (boots <= 0) return cudaSuccess;
    switch (p.N) {
        case 512: return launch_br_n<512>(precision, bsk, bara, bara_stride, boots, nsteps, mu, acc_in, acc_out, p.Bgbit, s, gpb);
        case 1024: return launch_br_n<1024>(precision, bsk, bara, bara_stride, boots, nsteps, mu, acc_in, acc_out, p.Bgbit, s, gpb);
        case 2048: return launch_br_n<2048>(precision, bsk, bara, bara_stride, boots, nsteps, mu, acc_in, acc_out, p.Bgbit, s, gpb);
        default: return cudaErrorInvalidValue;
    }
}

// ============================================================================================
// sample extraction (+ MUX recombination)
// ============================================================================================

// one CTA per gate; out row = extract(acc[boot0]) (+ extract(acc[boot1])) + (0, cst)
__global__ void extract_kernel(const GateDesc *__restrict__ desc, const uint32_t *__restrict__ acc, int N, int k,
                               uint32_t *__restrict__ out, int out_stride) {
    const GateDesc d = desc[blockIdx.x];
    const int kN = k * N;
    const size_t tl = (size_t)(k + 1) * N;
    const uint32_t *a0 = acc + (size_t)d.boot0 * tl;
    const uint32_t *a1 = d.boot1 >= 0 ? acc + (size_t)d.boot1 * tl : nullptr;
    uint32_t *o = out + (size_t)blockIdx.x * out_stride;
    for (int i = threadIdx.x; i <= kN; i += blockDim.x) {
        // lwe.cpp:46-52: a'[u*N+0] = a_u[0], a'[u*N+j] = -a_u[N-j], b' = b[0]
        uint32_t v;
        if (i == kN) {
            v = a0[kN];
            if (a1) v += a1[kN];
            v += (uint32_t)d.cst;
        } else {
            const int u = i / N, j = i - u * N;
            const size_t src = (size_t)u * N + (j == 0 ? 0 : N - j);
            v = a0[src];
            if (a1) v += a1[src];
            if (j != 0) v = 0u - v;
        }
        o[i] = v;
    }
}

cudaError_t launch_extract(const tfheb_params &p, const GateDesc *d_desc, int count, const int32_t *acc,
                           int32_t *out, int out_stride, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    extract_kernel<<<count, 256, 0, s>>>(d_desc, reinterpret_cast<const uint32_t *>(acc), p.N, p.k,
                                         reinterpret_cast<uint32_t *>(out), out_stride);
    return cudaGetLastError();
}

__global__ void negate_kernel(const uint32_t *__restrict__ in, uint32_t *__restrict__ out, size_t count) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x)
        out[i] = 0u - in[i];
}

// bootsNOT (boot-gates.cpp:164-167): elementwise negation of the ciphertexts
cudaError_t launch_negate(const int32_t *in, int32_t *out, size_t count, cudaStream_t s) {
    if (count == 0) return cudaSuccess;
    const int blocks = (int)std::min<size_t>((count + 255) / 256, 148 * 8);
    negate_kernel<<<blocks, 256, 0, s>>>(reinterpret_cast<const uint32_t *>(in), reinterpret_cast<uint32_t *>(out),
                                         count);
    return cudaGetLastError();
}

// ============================================================================================
// keyswitch
// ============================================================================================

// One CTA per gate; thread owns 4 consecutive output coefficients (int4 loads of the key rows).
// ksk rows: [kN][t][base][ks_stride], ks_stride a multiple of 4, zero padded.
__global__ void __launch_bounds__(256) keyswitch_kernel(const int32_t *__restrict__ ksk, int ks_stride,
                                                        const uint32_t *__restrict__ in, int in_stride,
                                                        uint32_t *__restrict__ out, int n, int kN, int t,
                                                        int basebit) {
    const int g = blockIdx.x;
    const uint32_t *x = in + (size_t)g * in_stride;
    const int c4 = threadIdx.x * 4;
    const bool active = c4 < ks_stride;
    const int base = 1 << basebit;
    const uint32_t mask = (uint32_t)base - 1;
    const uint32_t prec_offset = 1u << (32 - (1 + basebit * t));  // lwe-keyswitch-functions.cpp:119
    uint32_t acc0 = 0, acc1 = 0, acc2 = 0, acc3 = 0;
    extern __shared__ uint32_t s_a[];  // the input mask, kN values
    for (int i = threadIdx.x; i < kN; i += blockDim.x) s_a[i] = x[i] + prec_offset;
    __syncthreads();
    if (active) {
        const size_t row_i = (size_t)t * base * ks_stride;
        for (int i = 0; i < kN; i++) {
            const uint32_t aibar = s_a[i];
            const int4 *rows = reinterpret_cast<const int4 *>(ksk + (size_t)i * row_i) + (c4 >> 2);
            for (int j = 0; j < t; j++) {
                const uint32_t aij = (aibar >> (32 - (j + 1) * basebit)) & mask;
                if (aij != 0) {
                    const int4 v = __ldg(rows + ((size_t)(j * base + aij) * ks_stride >> 2));
                    acc0 -= (uint32_t)v.x;
                    acc1 -= (uint32_t)v.y;
                    acc2 -= (uint32_t)v.z;
                    acc3 -= (uint32_t)v.w;
                }
            }
        }
        // result = (0, b) - sum  (lwe-keyswitch-functions.cpp:233-237)
        uint32_t *o = out + (size_t)g * (n + 1);
        const uint32_t b = x[kN];
        const uint32_t accs[4] = {acc0, acc1, acc2, acc3};
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const int col = c4 + e;
            if (col < n) o[col] = accs[e];
            else if (col == n) o[col] = b + accs[e];
        }
    }
}

cudaError_t launch_keyswitch(const tfheb_params &p, const int32_t *d_ksk, int ks_stride, int count,
                             const int32_t *in, int in_stride, int32_t *out, cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    const int kN = p.k * p.N;
    const int threads = ((ks_stride / 4 + 31) / 32) * 32;
    if (threads > 256) return cudaErrorInvalidValue;
    keyswitch_kernel<<<count, threads, sizeof(uint32_t) * kN, s>>>(
        d_ksk, ks_stride, reinterpret_cast<const uint32_t *>(in), in_stride, reinterpret_cast<uint32_t *>(out), p.n,
        kN, p.ks_t, p.ks_basebit);
    return cudaGetLastError();
}

// ============================================================================================
// FMA throughput probe: the FP32 / FP64 CUDA-core roofline denominator of the blind rotation,
// measured on the running GPU at its current clocks (8 independent FMA chains per thread).
// ============================================================================================

template <typename T>
__global__ void fma_peak_kernel(T *out, int iters, T a, T b) {
    T x0 = T(threadIdx.x), x1 = x0 + T(1), x2 = x0 + T(2), x3 = x0 + T(3);
    T x4 = x0 + T(4), x5 = x0 + T(5), x6 = x0 + T(6), x7 = x0 + T(7);
    for (int i = 0; i < iters; i++) {
        x0 = fma(x0, a, b); x1 = fma(x1, a, b); x2 = fma(x2, a, b); x3 = fma(x3, a, b);
        x4 = fma(x4, a, b); x5 = fma(x5, a, b); x6 = fma(x6, a, b); x7 = fma(x7, a, b);
    }
    const T s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == T(-1234.5)) out[0] = s;  // keeps the chains live
}

cudaError_t measure_fma_peak(int precision, double *tflops) {
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const int blocks = sms * 8, threads = 256, iters = 1 << 14;
    void *out = nullptr;
    cudaError_t e = cudaMalloc(&out, 16);
    if (e != cudaSuccess) return e;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    for (int rep = 0; rep < 4; rep++) {
        cudaEventRecord(e0);
        if (precision == TFHEB_FP64)
            fma_peak_kernel<double><<<blocks, threads>>>((double *)out, iters, 0.999999, 1e-7);
        else
            fma_peak_kernel<float><<<blocks, threads>>>((float *)out, iters, 0.9999f, 1e-7f);
        cudaEventRecord(e1);
        cudaEventSynchronize(e1);
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        if (rep > 0) best = std::min(best, ms);
    }
    e = cudaGetLastError();
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    *tflops = 2.0 * 8.0 * iters * (double)blocks * threads / (best * 1e-3) / 1e12;
    return e;
}

}  // namespace tfheb
