// br_common.cuh -- pieces shared by the blind-rotation kernels (blind_rotate.cu,
// blind_rotate_paired.cu): launch arguments, the exact integer/float conversions and the
// (X^a - 1) rotation.  Every kernel computes these the same way, so all give the same bits.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tfheb {

struct BrArgs {
    const int32_t *bara;
    int bara_stride;
    const uint8_t *bsk;
    const void *tables;
    const void *tables2;  // split-FP32 twiddles as broadcast pairs (the paired kernel)
    const int32_t *acc_in;
    int32_t *acc_out;
    int boots, nsteps;
    int32_t mu;
    int Bgbit;
    int split_shift;
    int32_t *err;
    uint64_t timeout_ns;
    int stall_producer;
};

// ---- exact conversions without the conversion (XU) pipe ------------------------------------

// small non-negative integer d (d < 2^22) -> float d - (bias - 1.5*2^23): the bits of 1.5*2^23 + d are
// 0x4B400000 | d, so the digit mask and this OR fuse into one logic op
__device__ __forceinline__ float biased_to_float(uint32_t d, float bias) {
    return __int_as_float(0x4B400000u | d) - bias;
}
// round-to-nearest of a float with |v| < 2^44, reduced mod 2^32 (FMA/ALU ops only)
__device__ __forceinline__ uint32_t round_f32_mod32(float v) {
    const float magic = 12582912.0f;  // 1.5 * 2^23
    const float m1 = fmaf(v, 0x1.0p-22f, magic);
    const uint32_t th = (uint32_t)(__float_as_int(m1) - 0x4B400000);
    const float r = fmaf(-(m1 - magic), 4194304.0f, v);  // exact: |r| <= 2^21
    const uint32_t tl = (uint32_t)(__float_as_int(r + magic) - 0x4B400000);
    return (th << 22) + tl;
}
// round-to-nearest of a double with |v| < 2^51, reduced mod 2^32
__device__ __forceinline__ uint32_t round_f64_mod32(double v) {
    return (uint32_t)__double2loint(v + 6755399441055744.0);  // 1.5 * 2^52
}

template <typename T>
struct DigitConv;
template <>
struct DigitConv<float> {
    // value d - halfBg of a raw digit d in [0, Bg)
    __device__ __forceinline__ static float conv(uint32_t d, float bias) { return biased_to_float(d, bias); }
    __host__ __device__ static constexpr float base() { return 12582912.0f; }
};
template <>
struct DigitConv<double> {
    __device__ __forceinline__ static double conv(uint32_t d, double bias) {
        return __hiloint2double(0x43380000, (int)d) - bias;
    }
    __host__ __device__ static constexpr double base() { return 6755399441055744.0; }
};

// (X^a - 1) * acc, coefficient j (toruspolynomial-functions.cpp:117-136), 0 <= a < 2N, without
// branches: e = (j - a) mod 2N selects coefficient e mod N, negated when e >= N (X^N = -1).
template <int N>
__device__ __forceinline__ uint32_t rot_minus_one(const uint32_t *poly, int j, int a) {
    const int e = (j - a) & (2 * N - 1);
    const uint32_t neg = 0u - (uint32_t)((e & N) != 0);
    return ((poly[e & (N - 1)] ^ neg) - neg) - poly[j];
}

}  // namespace tfheb
