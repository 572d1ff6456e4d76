// fft.cuh -- negacyclic FFT building blocks for the blind-rotation kernel (sm_100a).
//
// A real polynomial a of degree < N in R[X]/(X^N+1) is folded into M = N/2 complex points
//     z_j = (a_j - i a_{j+M}) * exp(-i pi j / N),   j < M,
// and a size-M complex DFT with W = exp(-2 pi i / M) then evaluates a at the M primitive 2N-th
// roots exp(-i pi (4k+1) / N); products in the ring become pointwise products.  This is the same
// "half-size complex" representation the reference keeps in LagrangeHalfCPolynomial
// (fft_processors/spqlios/lagrangehalfc_impl.h:40-45), derived and laid out independently here.
//
// One FFT is computed by a team of T = M/R threads holding R = 8 points each in registers.
// The transform is an in-place mixed-radix decimation-in-frequency over the stage radices of
// FftPlan<M>; between stages the team exchanges points through shared memory.  The forward
// transform leaves the spectrum in "slot order" (thread t, register r) = digit-reversed frequency,
// so no reordering pass exists: the bootstrapping key is stored in the same slot order by the host,
// the multiply-accumulate is pointwise on registers, and the inverse transform (the exact adjoint
// of the forward stages) consumes slot order and returns natural order.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace tfheb {

template <typename T>
struct cplx {
    T re, im;
};

template <typename T>
__device__ __forceinline__ cplx<T> cadd(cplx<T> a, cplx<T> b) { return {a.re + b.re, a.im + b.im}; }
template <typename T>
__device__ __forceinline__ cplx<T> csub(cplx<T> a, cplx<T> b) { return {a.re - b.re, a.im - b.im}; }
template <typename T>
__device__ __forceinline__ cplx<T> cmul(cplx<T> a, cplx<T> b) {
    return {fma(a.re, b.re, -a.im * b.im), fma(a.re, b.im, a.im * b.re)};
}
template <typename T>
__device__ __forceinline__ cplx<T> cmulconj(cplx<T> a, cplx<T> b) {  // a * conj(b)
    return {fma(a.re, b.re, a.im * b.im), fma(a.im, b.re, -a.re * b.im)};
}
// acc += a * b
template <typename T>
__device__ __forceinline__ void cmac(cplx<T> &acc, cplx<T> a, cplx<T> b) {
    acc.re = fma(a.re, b.re, acc.re);
    acc.re = fma(-a.im, b.im, acc.re);
    acc.im = fma(a.re, b.im, acc.im);
    acc.im = fma(a.im, b.re, acc.im);
}

// multiply by -i (forward) or +i (inverse)
template <typename T, bool INV>
__device__ __forceinline__ cplx<T> rot_quarter(cplx<T> a) {
    if (INV) return {-a.im, a.re};
    return {a.im, -a.re};
}

template <typename T>
__device__ __forceinline__ T rsqrt2() { return T(0.70710678118654752440084436210485); }

// ---- small DFT codelets: natural-order input and output, W_r = exp(-2 pi i / r) (conj if INV) --

template <typename T, bool INV>
__device__ __forceinline__ void dft2(cplx<T> *x) {
    const cplx<T> a = x[0], b = x[1];
    x[0] = cadd(a, b);
    x[1] = csub(a, b);
}

template <typename T, bool INV>
__device__ __forceinline__ void dft4(cplx<T> &x0, cplx<T> &x1, cplx<T> &x2, cplx<T> &x3) {
    const cplx<T> s02 = cadd(x0, x2), d02 = csub(x0, x2);
    const cplx<T> s13 = cadd(x1, x3), d13 = rot_quarter<T, INV>(csub(x1, x3));
    x0 = cadd(s02, s13);
    x2 = csub(s02, s13);
    x1 = cadd(d02, d13);
    x3 = csub(d02, d13);
}

template <typename T, bool INV>
__device__ __forceinline__ void dft4(cplx<T> *x) { dft4<T, INV>(x[0], x[1], x[2], x[3]); }

template <typename T, bool INV>
__device__ __forceinline__ void dft8(cplx<T> *x) {
    cplx<T> e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6];
    cplx<T> o0 = x[1], o1 = x[3], o2 = x[5], o3 = x[7];
    dft4<T, INV>(e0, e1, e2, e3);
    dft4<T, INV>(o0, o1, o2, o3);
    const T h = rsqrt2<T>();
    // o_k *= W8^k (forward W8 = (1-i)/sqrt2; inverse uses the conjugate); the 1/sqrt2 scaling is
    // folded into the combining additions as fused multiply-adds: w_k = h * (u_k + i v_k)
    T u1, v1, u3, v3;
    if (!INV) {
        u1 = o1.re + o1.im;
        v1 = o1.im - o1.re;
        u3 = o3.im - o3.re;
        v3 = -(o3.re + o3.im);
    } else {
        u1 = o1.re - o1.im;
        v1 = o1.re + o1.im;
        u3 = -(o3.re + o3.im);
        v3 = o3.re - o3.im;
    }
    const cplx<T> w2 = rot_quarter<T, INV>(o2);
    x[0] = cadd(e0, o0);
    x[4] = csub(e0, o0);
    x[1] = {fma(u1, h, e1.re), fma(v1, h, e1.im)};
    x[5] = {fma(-u1, h, e1.re), fma(-v1, h, e1.im)};
    x[2] = cadd(e2, w2);
    x[6] = csub(e2, w2);
    x[3] = {fma(u3, h, e3.re), fma(v3, h, e3.im)};
    x[7] = {fma(-u3, h, e3.re), fma(-v3, h, e3.im)};
}

template <typename T, bool INV, int RADIX>
__device__ __forceinline__ void dft(cplx<T> *x) {
    if constexpr (RADIX == 8) dft8<T, INV>(x);
    else if constexpr (RADIX == 4) dft4<T, INV>(x);
    else dft2<T, INV>(x);
}

// ---- packed FP32 (sm_100 f32x2): two complex numbers per register pair ------------------------
// A "cpair" holds two complex numbers in planar form, re = {a.re, b.re}, im = {a.im, b.im}.  Each
// packed instruction performs the two correctly rounded scalar operations, so packed code gives bit
// for bit the results of the scalar code with half the issued FP32 instructions.  The blind
// rotation uses it for the multiply-accumulate against the key; packing the FFT codelets as well
// measured slower (register-pair moves and longer dependency chains outweigh the saved issues).

struct cpair {
    float2 re, im;
};

__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

__device__ __forceinline__ cpair make_cpair(cplx<float> a, cplx<float> b) { return {{a.re, b.re}, {a.im, b.im}}; }

// acc += z * k on a register pair, with the scalar cmac operation order; nzi = -z.im, k = float4
// {re, re', im, im'}
__device__ __forceinline__ void cmac_pair(cpair &acc, const cpair &z, float2 nzi, float4 k) {
    const float2 kr{k.x, k.y}, ki{k.z, k.w};
    acc.re = fma2(z.re, kr, acc.re);
    acc.re = fma2(nzi, ki, acc.re);
    acc.im = fma2(z.re, ki, acc.im);
    acc.im = fma2(z.im, kr, acc.im);
}

// ---- plans -----------------------------------------------------------------------------------
// Stage radices per transform size (R = 8 points per thread): every radix divides R.

template <int M>
struct FftPlan;
template <>
struct FftPlan<64> {
    static constexpr int NS = 2;
    __host__ __device__ static constexpr int radix(int) { return 8; }
};
template <>
struct FftPlan<256> {
    static constexpr int NS = 3;
    __host__ __device__ static constexpr int radix(int s) { return s < 2 ? 8 : 4; }
};
template <>
struct FftPlan<512> {
    static constexpr int NS = 3;
    __host__ __device__ static constexpr int radix(int) { return 8; }
};
template <>
struct FftPlan<1024> {
    static constexpr int NS = 4;
    __host__ __device__ static constexpr int radix(int s) { return s < 3 ? 8 : 2; }
};

// sub-transform length entering stage S
template <int M>
__host__ __device__ constexpr int stage_len(int S) {
    int L = M;
    for (int s = 0; s < S; s++) L /= FftPlan<M>::radix(s);
    return L;
}

template <int M, int S>
struct Stage {
    static constexpr int r = FftPlan<M>::radix(S);
    static constexpr int L = stage_len<M>(S);
    static constexpr int stride = L / r;
};

// Twiddle tables, packed per stage.  Stage 0 stores the combined factor
//     exp(-i pi t / N) * W_M^{t*k2}   at [k2*NT + t], k2 in [0, 8)
// (the negacyclic twist exp(-i pi j / N), j = t + NT*n2, split as exp(-i pi t/N) * exp(-i pi n2/16):
// the first factor is common to the thread's eight inputs and moves behind the radix-8 DFT, the
// second is a compile-time constant applied before it).  Stages S >= 1 store W_L^{n1*k2} at
// [(k2-1)*stride + n1], k2 in [1, r), n1 < stride.
template <int M>
__host__ __device__ constexpr int tw_offset(int S) {
    int off = 0;
    for (int s = 0; s < S; s++) {
        const int L = stage_len<M>(s), r = FftPlan<M>::radix(s);
        off += (s == 0 ? r : r - 1) * (L / r);
    }
    return off;
}

// FP32 twiddle table, in float4 pairs so that one 16-byte load feeds two registers.  Stage S (radix r,
// stride st = L/r) holds r/2 float4 per n1 < st at [p][st]: stage 0 pairs {w(2p), w(2p+1)} of the
// factors above (k2 = 2p, 2p+1; st = NT), stages S >= 1 pairs {w(2p+1), w(2p+2)} (k2 = 2p+1, 2p+2; an
// odd count ends with a zero pad).  Offsets in float4 units.
template <int M>
__host__ __device__ constexpr int tw4_offset(int S) {
    int off = 0;
    for (int s = 0; s < S; s++) off += (FftPlan<M>::radix(s) / 2) * (stage_len<M>(s) / FftPlan<M>::radix(s));
    return off;
}
// bytes of the twiddle table of a T transform (a multiple of 16)
template <typename T, int M>
__host__ __device__ constexpr int tw_table_bytes() {
    return sizeof(T) == 4 ? 16 * tw4_offset<M>(FftPlan<M>::NS) : 16 * tw_offset<M>(FftPlan<M>::NS);
}

// exp(-i pi n / 16), n = 0..7: the per-register part of the twist (NT / N = 1/16 for R = 8)
__host__ __device__ constexpr double fold_cos(int n) {
    return n == 0 ? 1.0 : n == 1 ? 0.98078528040323044913 : n == 2 ? 0.92387953251128675613
         : n == 3 ? 0.83146961230254523708 : n == 4 ? 0.70710678118654752440 : n == 5 ? 0.55557023301960222474
         : n == 6 ? 0.38268343236508977173 : 0.19509032201612826785;
}
__host__ __device__ constexpr double fold_sin(int n) { return n == 0 ? 0.0 : fold_cos(8 - n); }

// Exchange buffers of one team FFT (M complex points).  Exchange E moves the points from stage E's
// registers to stage E+1's (the inverse runs the same exchanges backwards); its layout maps point p
// to an element index.  Every layout is separable on both of its stages: the index of a thread's
// register (c, n2) is the thread's base index combined with a compile-time constant, by addition
// (the constant folds into the load/store offset) or, for the XOR swizzle, by one XOR per access.
// TeamFft asserts both properties at compile time.
//   double: interleaved double2 with one pad element every 8, p + (p >> 3), for every exchange;
//           simulated over all stores and loads of the 8*8*8 and 8*8*8*2 plans, conflict free for
//           16-byte accesses.
//   float:  interleaved float2, one map per exchange.  An 8-byte warp access is served as two
//           half-warp wavefronts, each costing the largest number of distinct 8-byte words on one of
//           the 16 bank pairs; this model matched the wavefronts measured on B200 for 12 candidate
//           maps of the 8*8*8 plan.  The maps below reach the minimum of two wavefronts per access on
//           both stages of their exchange, padded (additive) where such a padding exists and
//           XOR-swizzled p ^ ((p >> 2) & 7) ^ ((p >> 3) & 31) on the last exchange of the 8*8*8*2
//           plan, where none does.  A single map for all exchanges (the swizzle) costs a XOR per
//           access; p + (p >> 3) for all of them costs 2.5 wavefronts per access.
struct ExchMap {
    int s1, a, s2, b;  // index = p + a * (p >> s1) + b * (p >> s2)
    bool swizzle;      // index = p ^ ((p >> 2) & 7) ^ ((p >> 3) & 31) instead
};
template <int M>
__host__ __device__ constexpr ExchMap exch_f32_map(int E) {
    return M == 256    ? (E == 0 ? ExchMap{5, 4, 6, 0, false} : ExchMap{2, 1, 6, 4, false})
           : M == 512  ? (E == 0 ? ExchMap{5, 4, 6, 0, false} : ExchMap{3, 1, 4, 0, false})
           : M == 1024 ? (E == 0   ? ExchMap{2, 0, 3, 0, false}
                          : E == 1 ? ExchMap{4, 2, 5, 0, false}
                                   : ExchMap{0, 0, 0, 0, true})
                       : ExchMap{2, 0, 3, 0, false};
}
template <int M>
__host__ __device__ constexpr int exch_f32_index(int E, int p) {
    const ExchMap m = exch_f32_map<M>(E);
    return m.swizzle ? p ^ ((p >> 2) & 7) ^ ((p >> 3) & 31) : p + m.a * (p >> m.s1) + m.b * (p >> m.s2);
}
template <int M>
__host__ __device__ constexpr int exch_f32_slots() {
    int n = 0;
    for (int E = 0; E + 1 < FftPlan<M>::NS; E++)
        for (int p = 0; p < M; p++) n = n > exch_f32_index<M>(E, p) + 1 ? n : exch_f32_index<M>(E, p) + 1;
    return n;
}

template <typename T, int M>
struct Exch;
template <int M>
struct Exch<double, M> {
    static constexpr int slots = M + (M >> 3);
    static constexpr int bytes = 16 * slots;
    __host__ __device__ static constexpr bool additive(int) { return true; }
    __host__ __device__ static constexpr int index(int, int p) { return p + (p >> 3); }
    __device__ static __forceinline__ void put(void *buf, int i, cplx<double> v) {
        reinterpret_cast<cplx<double> *>(buf)[i] = v;
    }
    __device__ static __forceinline__ cplx<double> get(const void *buf, int i) {
        return reinterpret_cast<const cplx<double> *>(buf)[i];
    }
};
template <int M>
struct Exch<float, M> {
    static constexpr int slots = exch_f32_slots<M>();
    static constexpr int bytes = 8 * slots;
    __host__ __device__ static constexpr bool additive(int E) { return !exch_f32_map<M>(E).swizzle; }
    __host__ __device__ static constexpr int index(int E, int p) { return exch_f32_index<M>(E, p); }
    __device__ static __forceinline__ void put(void *buf, int i, cplx<float> v) {
        reinterpret_cast<float2 *>(buf)[i] = make_float2(v.re, v.im);
    }
    __device__ static __forceinline__ cplx<float> get(const void *buf, int i) {
        const float2 v = reinterpret_cast<const float2 *>(buf)[i];
        return {v.x, v.y};
    }
};

// Named barrier over one team (ids 1..15; 0 is __syncthreads).
__device__ __forceinline__ void team_sync(int id, int nthreads) {
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(nthreads) : "memory");
}

// Exchange buffers of a team.  With two (stride = bytes of one buffer) consecutive exchanges
// alternate between them (the parity runs on across transforms): exchange k stores into buffer
// k % 2, whose last readers (exchange k-2) all passed the barrier of exchange k-1 before this store,
// so one barrier per exchange suffices.  With one (stride = 0) every exchange ends with a second
// barrier before the buffer is reused; variants short of shared memory or registers use that.
struct ExchPair {
    unsigned char *base;
    uint32_t stride;  // bytes of one buffer; 0: a single buffer
    uint32_t parity;  // buffer of the next exchange
    __device__ __forceinline__ void *next() {
        void *b = base + parity * stride;
        parity ^= 1u;
        return b;
    }
};

// Team FFT: T = M/R threads, t in [0,T), registers x[R], one or two exchange buffers (ExchPair).
template <typename T, int M, int R>
struct TeamFft {
    static constexpr int NT = M / R;  // threads per team
    static constexpr int NS = FftPlan<M>::NS;
    static_assert(R == 8 && FftPlan<M>::radix(0) == 8, "stage 0 is the thread's own radix-8 DFT");

    // position of register (c, n2) of thread t at stage S
    template <int S>
    __host__ __device__ static constexpr int pos(int t, int c, int n2) {
        constexpr int L = Stage<M, S>::L, st = Stage<M, S>::stride;
        const int b = t + NT * c;
        const int q = b / st, n1 = b - q * st;
        return q * L + n1 + st * n2;
    }
    // index of point p in exchange E's buffer; base index combined with a compile-time constant
    __host__ __device__ static constexpr int xindex(int E, int p) { return Exch<T, M>::index(E, p); }
    __host__ __device__ static constexpr int xcombine(int E, int base, int d) {
        return Exch<T, M>::additive(E) ? base + d : base ^ d;
    }
    // compile-time part of the index of register (c, n2) at stage S in exchange E (pos<S>(0,0,0) = 0)
    template <int S, int E>
    __host__ __device__ static constexpr int delta(int c, int n2) {
        return Exch<T, M>::additive(E) ? xindex(E, pos<S>(0, c, n2)) - xindex(E, 0)
                                       : xindex(E, pos<S>(0, c, n2)) ^ xindex(E, 0);
    }

    // Every exchange layout must be a one-to-one map of the M positions into the buffer, and on both
    // of its stages each register's index must be the thread's base index combined with a constant.
    static constexpr bool exchange_layout_valid() {
        using X = Exch<T, M>;
        for (int E = 0; E + 1 < NS; E++) {
            bool seen[X::slots] = {};
            for (int p = 0; p < M; p++) {
                const int i = xindex(E, p);
                if (i < 0 || i >= X::slots || seen[i]) return false;
                seen[i] = true;
            }
            for (int S = E; S <= E + 1; S++) {
                const int L = stage_len<M>(S), r = FftPlan<M>::radix(S), st = L / r;
                for (int t = 0; t < NT; t++)
                    for (int c = 0; c < R / r; c++)
                        for (int n2 = 0; n2 < r; n2++) {
                            const int b0 = NT * c, b = t + NT * c;
                            const int p0 = (b0 / st) * L + b0 % st + st * n2;
                            const int p = (b / st) * L + b % st + st * n2;
                            const int t0 = (t / st) * L + t % st;
                            const int d = X::additive(E) ? xindex(E, p0) - xindex(E, 0) : xindex(E, p0) ^ xindex(E, 0);
                            if (xcombine(E, xindex(E, t0), d) != xindex(E, p)) return false;
                        }
            }
        }
        return true;
    }

    // stage S's registers to / from exchange E's buffer
    template <int S, int E>
    __device__ static __forceinline__ void store(const cplx<T> *x, void *buf, int t) {
        static_assert(exchange_layout_valid(), "exchange layout not one-to-one or not separable on some stage");
        constexpr int r = Stage<M, S>::r;
        const int base = xindex(E, pos<S>(t, 0, 0));
#pragma unroll
        for (int c = 0; c < R / r; c++)
#pragma unroll
            for (int n2 = 0; n2 < r; n2++)
                Exch<T, M>::put(buf, xcombine(E, base, delta<S, E>(c, n2)), x[c * r + n2]);
    }

    template <int S, int E>
    __device__ static __forceinline__ void load(cplx<T> *x, const void *buf, int t) {
        constexpr int r = Stage<M, S>::r;
        const int base = xindex(E, pos<S>(t, 0, 0));
#pragma unroll
        for (int c = 0; c < R / r; c++)
#pragma unroll
            for (int n2 = 0; n2 < r; n2++)
                x[c * r + n2] = Exch<T, M>::get(buf, xcombine(E, base, delta<S, E>(c, n2)));
    }

    template <int S, bool INV>
    __device__ static __forceinline__ void twiddle(cplx<T> *x, const cplx<T> *tw, int t) {
        constexpr int r = Stage<M, S>::r, st = Stage<M, S>::stride;
        if constexpr (sizeof(T) == 4) {  // paired float4 table (tw4_offset)
            const float4 *tw4 = reinterpret_cast<const float4 *>(tw) + tw4_offset<M>(S);
            auto apply = [&](cplx<T> &v, float re, float im) {
                const cplx<T> w{re, im};
                v = INV ? cmulconj(v, w) : cmul(v, w);
            };
            if constexpr (S == 0) {
#pragma unroll
                for (int q = 0; q < r / 2; q++) {
                    const float4 w = tw4[q * NT + t];
                    apply(x[2 * q], w.x, w.y);
                    apply(x[2 * q + 1], w.z, w.w);
                }
            } else if constexpr (st > 1) {
#pragma unroll
                for (int c = 0; c < R / r; c++) {
                    const int n1 = (t + NT * c) % st;
#pragma unroll
                    for (int q = 0; q < r / 2; q++) {
                        const float4 w = tw4[q * st + n1];
                        apply(x[c * r + 2 * q + 1], w.x, w.y);
                        if (2 * q + 2 < r) apply(x[c * r + 2 * q + 2], w.z, w.w);
                    }
                }
            }
        } else if constexpr (S == 0) {
#pragma unroll
            for (int k2 = 0; k2 < r; k2++) {
                const cplx<T> w = tw[k2 * NT + t];
                x[k2] = INV ? cmulconj(x[k2], w) : cmul(x[k2], w);
            }
        } else if constexpr (st > 1) {
            const cplx<T> *tws = tw + tw_offset<M>(S);
#pragma unroll
            for (int c = 0; c < R / r; c++) {
                const int b = t + NT * c;
                const int n1 = b % st;
#pragma unroll
                for (int k2 = 1; k2 < r; k2++) {
                    const cplx<T> w = tws[(k2 - 1) * st + n1];
                    x[c * r + k2] = INV ? cmulconj(x[c * r + k2], w) : cmul(x[c * r + k2], w);
                }
            }
        }
    }

    // x[n] *= exp(-+ i pi n / 16)
    template <bool INV>
    __device__ static __forceinline__ void fold_consts(cplx<T> *x) {
#pragma unroll
        for (int n = 1; n < R; n++) {
            const cplx<T> w{T(fold_cos(n)), T(-fold_sin(n))};
            x[n] = INV ? cmulconj(x[n], w) : cmul(x[n], w);
        }
    }

    template <int S>
    __device__ static __forceinline__ void forward_from(cplx<T> *x, ExchPair &xp, const cplx<T> *tw, int t, int bar_id) {
        constexpr int r = Stage<M, S>::r;
#pragma unroll
        for (int c = 0; c < R / r; c++) dft<T, false, r>(x + c * r);
        twiddle<S, false>(x, tw, t);
        if constexpr (S + 1 < NS) {
            void *buf = xp.next();
            store<S, S>(x, buf, t);
            team_sync(bar_id, NT);
            load<S + 1, S>(x, buf, t);
            if (xp.stride == 0) team_sync(bar_id, NT);
            forward_from<S + 1>(x, xp, tw, t, bar_id);
        }
    }

    template <int S>
    __device__ static __forceinline__ void inverse_from(cplx<T> *x, ExchPair &xp, const cplx<T> *tw, int t, int bar_id) {
        constexpr int r = Stage<M, S>::r;
        twiddle<S, true>(x, tw, t);
#pragma unroll
        for (int c = 0; c < R / r; c++) dft<T, true, r>(x + c * r);
        if constexpr (S > 0) {
            void *buf = xp.next();
            store<S, S - 1>(x, buf, t);
            team_sync(bar_id, NT);
            load<S - 1, S - 1>(x, buf, t);
            if (xp.stride == 0) team_sync(bar_id, NT);
            inverse_from<S - 1>(x, xp, tw, t, bar_id);
        }
    }

    // Two independent forward transforms side by side, the counterpart of inverse_pair below (same
    // barriers, both buffers, parity untouched): each array goes through exactly the operations of
    // forward().  The caller's next exchange must begin with a barrier (forward_pair and
    // inverse_pair do).
    template <int S>
    __device__ static __forceinline__ void forward_pair_from(cplx<T> *x, cplx<T> *y, const ExchPair &xp,
                                                             const cplx<T> *tw, int t, int bar_id) {
        constexpr int r = Stage<M, S>::r;
#pragma unroll
        for (int c = 0; c < R / r; c++) {
            dft<T, false, r>(x + c * r);
            dft<T, false, r>(y + c * r);
        }
        twiddle<S, false>(x, tw, t);
        twiddle<S, false>(y, tw, t);
        if constexpr (S + 1 < NS) {
            unsigned char *bx = xp.base, *by = xp.base + xp.stride;
            store<S, S>(x, bx, t);
            store<S, S>(y, by, t);
            team_sync(bar_id, NT);
            load<S + 1, S>(x, bx, t);
            load<S + 1, S>(y, by, t);
            if constexpr (S + 2 < NS) team_sync(bar_id, NT);
            forward_pair_from<S + 1>(x, y, xp, tw, t, bar_id);
        }
    }
    __device__ static __forceinline__ void forward_pair(cplx<T> *x, cplx<T> *y, ExchPair &xp, const cplx<T> *tw, int t,
                                                        int bar_id) {
        fold_consts<false>(x);
        fold_consts<false>(y);
        team_sync(bar_id, NT);
        forward_pair_from<0>(x, y, xp, tw, t, bar_id);
    }

    // Two independent inverse transforms, stage by stage side by side: each array goes through
    // exactly the operations of inverse(), and the scheduler gets two dependency chains.  Every
    // exchange uses both exchange buffers (one per array), so a barrier precedes the first stores (the
    // other buffer may still be read by the previous exchange) and separates each exchange's loads
    // from the next one's stores.  Needs two buffers (xp.stride != 0).
    template <int S>
    __device__ static __forceinline__ void inverse_pair_from(cplx<T> *x, cplx<T> *y, const ExchPair &xp,
                                                             const cplx<T> *tw, int t, int bar_id) {
        constexpr int r = Stage<M, S>::r;
        twiddle<S, true>(x, tw, t);
        twiddle<S, true>(y, tw, t);
#pragma unroll
        for (int c = 0; c < R / r; c++) {
            dft<T, true, r>(x + c * r);
            dft<T, true, r>(y + c * r);
        }
        if constexpr (S > 0) {
            unsigned char *bx = xp.base, *by = xp.base + xp.stride;
            store<S, S - 1>(x, bx, t);
            store<S, S - 1>(y, by, t);
            team_sync(bar_id, NT);
            load<S - 1, S - 1>(x, bx, t);
            load<S - 1, S - 1>(y, by, t);
            if constexpr (S - 1 > 0) team_sync(bar_id, NT);
            inverse_pair_from<S - 1>(x, y, xp, tw, t, bar_id);
        }
    }
    __device__ static __forceinline__ void inverse_pair(cplx<T> *x, cplx<T> *y, ExchPair &xp, const cplx<T> *tw, int t,
                                                        int bar_id) {
        team_sync(bar_id, NT);
        inverse_pair_from<NS - 1>(x, y, xp, tw, t, bar_id);
        fold_consts<true>(x);
        fold_consts<true>(y);
    }

    // Folded negacyclic transform.  In: x[n2] = a_j - i a_{j+M} for j = t + NT*n2 (no twist applied).
    // Out: the M evaluation points in slot order.
    __device__ static __forceinline__ void forward(cplx<T> *x, ExchPair &xp, const cplx<T> *tw, int t, int bar_id) {
        fold_consts<false>(x);
        forward_from<0>(x, xp, tw, t, bar_id);
    }
    // Slot order in -> x[n2] = M * (c_j - i c_{j+M}), j = t + NT*n2 (twist removed).
    __device__ static __forceinline__ void inverse(cplx<T> *x, ExchPair &xp, const cplx<T> *tw, int t, int bar_id) {
        inverse_from<NS - 1>(x, xp, tw, t, bar_id);
        fold_consts<true>(x);
    }
};

// ---- two transforms per thread on packed f32x2 --------------------------------------------------
// TeamFft2 runs two independent FP32 transforms of the same size in lockstep: register r of a thread
// holds point r of transform A in the .x halves and of transform B in the .y halves of a cpair.
// Every packed instruction performs, on each half, the scalar operation that TeamFft<float> performs
// at the same place (same operands, same rounding, same order; negations are exact), so each
// transform's result is TeamFft<float>'s bit for bit, with half the FP32 instructions issued.
// Twiddles come from a table of broadcast pairs {w.re, w.re, w.im, w.im} holding the scalar FP32
// table's factors (tw2_entries: the FP64 table's layout, tw_offset); the exchange moves one 16-byte
// {A.re, B.re, A.im, B.im} per point under the 16-byte layout of Exch<double, M>.

__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    float2 d;
    asm("sub.rn.f32x2 %0, %1, %2;"
        : "=l"(*reinterpret_cast<unsigned long long *>(&d))
        : "l"(*reinterpret_cast<const unsigned long long *>(&a)), "l"(*reinterpret_cast<const unsigned long long *>(&b)));
    return d;
}
__device__ __forceinline__ float2 neg2(float2 a) { return mul2(a, make_float2(-1.f, -1.f)); }  // exact
__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }

__device__ __forceinline__ cpair padd(const cpair &a, const cpair &b) { return {add2(a.re, b.re), add2(a.im, b.im)}; }
__device__ __forceinline__ cpair psub(const cpair &a, const cpair &b) { return {sub2(a.re, b.re), sub2(a.im, b.im)}; }

// cmul / cmulconj of both halves by one factor w = (wr, wi) given as broadcast pairs, with nwi = -wi
// (x * (-y) = -(x * y) exactly, so the negated product costs no instruction)
__device__ __forceinline__ cpair pmul(const cpair &a, float2 wr, float2 wi, float2 nwi) {
    // {fma(a.re, w.re, -(a.im * w.im)), fma(a.re, w.im, a.im * w.re)}
    return {fma2(a.re, wr, mul2(a.im, nwi)), fma2(a.re, wi, mul2(a.im, wr))};
}
__device__ __forceinline__ cpair pmulconj(const cpair &a, float2 wr, float2 wi, float2 nwi) {
    // {fma(a.re, w.re, a.im * w.im), fma(a.im, w.re, -(a.re * w.im))}
    return {fma2(a.re, wr, mul2(a.im, wi)), fma2(a.im, wr, mul2(a.re, nwi))};
}

// dft4 of TeamFft on both halves; the quarter rotation is folded into which pair is added or
// subtracted (x + (-y) and x - y are the same IEEE operation)
template <bool INV>
__device__ __forceinline__ void pdft4(cpair &x0, cpair &x1, cpair &x2, cpair &x3) {
    const cpair s02 = padd(x0, x2), d02 = psub(x0, x2);
    const cpair s13 = padd(x1, x3), s = psub(x1, x3);
    x0 = padd(s02, s13);
    x2 = psub(s02, s13);
    if (!INV) {  // d13 = (s.im, -s.re)
        x1 = {add2(d02.re, s.im), sub2(d02.im, s.re)};
        x3 = {sub2(d02.re, s.im), add2(d02.im, s.re)};
    } else {     // d13 = (-s.im, s.re)
        x1 = {sub2(d02.re, s.im), add2(d02.im, s.re)};
        x3 = {add2(d02.re, s.im), sub2(d02.im, s.re)};
    }
}

template <bool INV>
__device__ __forceinline__ void pdft8(cpair *x) {
    cpair e0 = x[0], e1 = x[2], e2 = x[4], e3 = x[6];
    cpair o0 = x[1], o1 = x[3], o2 = x[5], o3 = x[7];
    pdft4<INV>(e0, e1, e2, e3);
    pdft4<INV>(o0, o1, o2, o3);
    const float2 h = bc2(rsqrt2<float>()), nh = bc2(-rsqrt2<float>());
    x[0] = padd(e0, o0);
    x[4] = psub(e0, o0);
    if (!INV) {
        // u1 = o1.re + o1.im, v1 = o1.im - o1.re, u3 = o3.im - o3.re, v3 = -(o3.re + o3.im)
        const float2 u1 = add2(o1.re, o1.im), v1 = sub2(o1.im, o1.re);
        const float2 u3 = sub2(o3.im, o3.re), p3 = add2(o3.re, o3.im);
        x[1] = {fma2(u1, h, e1.re), fma2(v1, h, e1.im)};
        x[5] = {fma2(u1, nh, e1.re), fma2(v1, nh, e1.im)};
        x[3] = {fma2(u3, h, e3.re), fma2(p3, nh, e3.im)};
        x[7] = {fma2(u3, nh, e3.re), fma2(p3, h, e3.im)};
        // w2 = (o2.im, -o2.re)
        x[2] = {add2(e2.re, o2.im), sub2(e2.im, o2.re)};
        x[6] = {sub2(e2.re, o2.im), add2(e2.im, o2.re)};
    } else {
        // u1 = o1.re - o1.im, v1 = o1.re + o1.im, u3 = -(o3.re + o3.im), v3 = o3.re - o3.im
        const float2 u1 = sub2(o1.re, o1.im), v1 = add2(o1.re, o1.im);
        const float2 p3 = add2(o3.re, o3.im), v3 = sub2(o3.re, o3.im);
        x[1] = {fma2(u1, h, e1.re), fma2(v1, h, e1.im)};
        x[5] = {fma2(u1, nh, e1.re), fma2(v1, nh, e1.im)};
        x[3] = {fma2(p3, nh, e3.re), fma2(v3, h, e3.im)};
        x[7] = {fma2(p3, h, e3.re), fma2(v3, nh, e3.im)};
        // w2 = (-o2.im, o2.re)
        x[2] = {sub2(e2.re, o2.im), add2(e2.im, o2.re)};
        x[6] = {add2(e2.re, o2.im), sub2(e2.im, o2.re)};
    }
}

template <int M>
struct TeamFft2 {
    static constexpr int R = 8, NT = M / R, NS = FftPlan<M>::NS;
    using Scalar = TeamFft<double, M, 8>;  // positions and the 16-byte exchange layout
    static_assert(FftPlan<M>::radix(0) == 8, "stage 0 is the thread's own radix-8 DFT");

    template <bool INV, int RADIX>
    __device__ static __forceinline__ void pdft(cpair *x) {
        if constexpr (RADIX == 8) pdft8<INV>(x);
        else if constexpr (RADIX == 4) pdft4<INV>(x[0], x[1], x[2], x[3]);
        else {
            const cpair a = x[0], b = x[1];
            x[0] = padd(a, b);
            x[1] = psub(a, b);
        }
    }

    template <int S, int E>
    __device__ static __forceinline__ void store(const cpair *x, void *buf, int t) {
        constexpr int r = Stage<M, S>::r;
        const int base = Scalar::xindex(E, Scalar::template pos<S>(t, 0, 0));
        float4 *b = reinterpret_cast<float4 *>(buf);
#pragma unroll
        for (int c = 0; c < R / r; c++)
#pragma unroll
            for (int n2 = 0; n2 < r; n2++) {
                const cpair &v = x[c * r + n2];
                b[base + Scalar::template delta<S, E>(c, n2)] = make_float4(v.re.x, v.re.y, v.im.x, v.im.y);
            }
    }
    template <int S, int E>
    __device__ static __forceinline__ void load(cpair *x, const void *buf, int t) {
        constexpr int r = Stage<M, S>::r;
        const int base = Scalar::xindex(E, Scalar::template pos<S>(t, 0, 0));
        const float4 *b = reinterpret_cast<const float4 *>(buf);
#pragma unroll
        for (int c = 0; c < R / r; c++)
#pragma unroll
            for (int n2 = 0; n2 < r; n2++) {
                const float4 v = b[base + Scalar::template delta<S, E>(c, n2)];
                x[c * r + n2] = {make_float2(v.x, v.y), make_float2(v.z, v.w)};
            }
    }

    // stage S's twiddles from the broadcast table (layout of tw_offset, one float4 per factor)
    template <int S, bool INV>
    __device__ static __forceinline__ void twiddle(cpair *x, const float4 *tw2, int t) {
        constexpr int r = Stage<M, S>::r, st = Stage<M, S>::stride;
        auto apply = [&](cpair &v, float4 w) {
            const float2 wr = make_float2(w.x, w.y), wi = make_float2(w.z, w.w);
            v = INV ? pmulconj(v, wr, wi, neg2(wi)) : pmul(v, wr, wi, neg2(wi));
        };
        if constexpr (S == 0) {
#pragma unroll
            for (int k2 = 0; k2 < r; k2++) apply(x[k2], tw2[k2 * NT + t]);
        } else if constexpr (st > 1) {
            const float4 *tws = tw2 + tw_offset<M>(S);
#pragma unroll
            for (int c = 0; c < R / r; c++) {
                const int n1 = (t + NT * c) % st;
#pragma unroll
                for (int k2 = 1; k2 < r; k2++) apply(x[c * r + k2], tws[(k2 - 1) * st + n1]);
            }
        }
    }

    // x[n] *= exp(-+ i pi n / 16): TeamFft::fold_consts with w = (cos, -sin) as float constants
    template <bool INV>
    __device__ static __forceinline__ void fold_consts(cpair *x) {
#pragma unroll
        for (int n = 1; n < R; n++) {
            const float wr = float(fold_cos(n)), wi = float(-fold_sin(n));
            x[n] = INV ? pmulconj(x[n], bc2(wr), bc2(wi), bc2(-wi)) : pmul(x[n], bc2(wr), bc2(wi), bc2(-wi));
        }
    }

    template <int S>
    __device__ static __forceinline__ void forward_from(cpair *x, ExchPair &xp, const float4 *tw2, int t, int bar_id) {
        constexpr int r = Stage<M, S>::r;
#pragma unroll
        for (int c = 0; c < R / r; c++) pdft<false, r>(x + c * r);
        twiddle<S, false>(x, tw2, t);
        if constexpr (S + 1 < NS) {
            void *buf = xp.next();
            store<S, S>(x, buf, t);
            team_sync(bar_id, NT);
            load<S + 1, S>(x, buf, t);
            if (xp.stride == 0) team_sync(bar_id, NT);
            forward_from<S + 1>(x, xp, tw2, t, bar_id);
        }
    }
    template <int S>
    __device__ static __forceinline__ void inverse_from(cpair *x, ExchPair &xp, const float4 *tw2, int t, int bar_id) {
        constexpr int r = Stage<M, S>::r;
        twiddle<S, true>(x, tw2, t);
#pragma unroll
        for (int c = 0; c < R / r; c++) pdft<true, r>(x + c * r);
        if constexpr (S > 0) {
            void *buf = xp.next();
            store<S, S - 1>(x, buf, t);
            team_sync(bar_id, NT);
            load<S - 1, S - 1>(x, buf, t);
            if (xp.stride == 0) team_sync(bar_id, NT);
            inverse_from<S - 1>(x, xp, tw2, t, bar_id);
        }
    }
    // TeamFft::forward on both halves.  In: x[n2] = a_j - i a_{j+M} of each transform.
    __device__ static __forceinline__ void forward(cpair *x, ExchPair &xp, const float4 *tw2, int t, int bar_id) {
        fold_consts<false>(x);
        forward_from<0>(x, xp, tw2, t, bar_id);
    }

    // Two independent forward() calls interleaved stage by stage: each stage's butterflies of x and y
    // are independent instruction chains, each twiddle factor is loaded once for both, and the two
    // exchanges of a stage share the buffer in turn.  Each array gets exactly forward()'s operations.
    template <int S>
    __device__ static __forceinline__ void twiddle_two(cpair *x, cpair *y, const float4 *tw2, int t) {
        constexpr int r = Stage<M, S>::r, st = Stage<M, S>::stride;
        auto apply = [&](cpair &v, cpair &u, float4 w) {
            const float2 wr = make_float2(w.x, w.y), wi = make_float2(w.z, w.w), nwi = neg2(wi);
            v = pmul(v, wr, wi, nwi);
            u = pmul(u, wr, wi, nwi);
        };
        if constexpr (S == 0) {
#pragma unroll
            for (int k2 = 0; k2 < r; k2++) apply(x[k2], y[k2], tw2[k2 * NT + t]);
        } else if constexpr (st > 1) {
            const float4 *tws = tw2 + tw_offset<M>(S);
#pragma unroll
            for (int c = 0; c < R / r; c++) {
                const int n1 = (t + NT * c) % st;
#pragma unroll
                for (int k2 = 1; k2 < r; k2++) apply(x[c * r + k2], y[c * r + k2], tws[(k2 - 1) * st + n1]);
            }
        }
    }
    template <int S>
    __device__ static __forceinline__ void forward_two_from(cpair *x, cpair *y, ExchPair &xp, const float4 *tw2, int t,
                                                            int bar_id) {
        constexpr int r = Stage<M, S>::r;
#pragma unroll
        for (int c = 0; c < R / r; c++) {
            pdft<false, r>(x + c * r);
            pdft<false, r>(y + c * r);
        }
        twiddle_two<S>(x, y, tw2, t);
        if constexpr (S + 1 < NS) {
            void *buf = xp.next();
            store<S, S>(x, buf, t);
            team_sync(bar_id, NT);
            load<S + 1, S>(x, buf, t);
            if (xp.stride == 0) team_sync(bar_id, NT);
            buf = xp.next();
            store<S, S>(y, buf, t);
            team_sync(bar_id, NT);
            load<S + 1, S>(y, buf, t);
            if (xp.stride == 0) team_sync(bar_id, NT);
            forward_two_from<S + 1>(x, y, xp, tw2, t, bar_id);
        }
    }
    __device__ static __forceinline__ void forward_two(cpair *x, cpair *y, ExchPair &xp, const float4 *tw2, int t,
                                                       int bar_id) {
        fold_consts<false>(x);
        fold_consts<false>(y);
        forward_two_from<0>(x, y, xp, tw2, t, bar_id);
    }
    // TeamFft::inverse on both halves.
    __device__ static __forceinline__ void inverse(cpair *x, ExchPair &xp, const float4 *tw2, int t, int bar_id) {
        inverse_from<NS - 1>(x, xp, tw2, t, bar_id);
        fold_consts<true>(x);
    }
    // Two independent inverse() calls interleaved stage by stage (as forward_two).
    template <int S>
    __device__ static __forceinline__ void twiddle_conj_two(cpair *x, cpair *y, const float4 *tw2, int t) {
        constexpr int r = Stage<M, S>::r, st = Stage<M, S>::stride;
        auto apply = [&](cpair &v, cpair &u, float4 w) {
            const float2 wr = make_float2(w.x, w.y), wi = make_float2(w.z, w.w), nwi = neg2(wi);
            v = pmulconj(v, wr, wi, nwi);
            u = pmulconj(u, wr, wi, nwi);
        };
        if constexpr (S == 0) {
#pragma unroll
            for (int k2 = 0; k2 < r; k2++) apply(x[k2], y[k2], tw2[k2 * NT + t]);
        } else if constexpr (st > 1) {
            const float4 *tws = tw2 + tw_offset<M>(S);
#pragma unroll
            for (int c = 0; c < R / r; c++) {
                const int n1 = (t + NT * c) % st;
#pragma unroll
                for (int k2 = 1; k2 < r; k2++) apply(x[c * r + k2], y[c * r + k2], tws[(k2 - 1) * st + n1]);
            }
        }
    }
    template <int S>
    __device__ static __forceinline__ void inverse_two_from(cpair *x, cpair *y, ExchPair &xp, const float4 *tw2, int t,
                                                            int bar_id) {
        constexpr int r = Stage<M, S>::r;
        twiddle_conj_two<S>(x, y, tw2, t);
#pragma unroll
        for (int c = 0; c < R / r; c++) {
            pdft<true, r>(x + c * r);
            pdft<true, r>(y + c * r);
        }
        if constexpr (S > 0) {
            void *buf = xp.next();
            store<S, S - 1>(x, buf, t);
            team_sync(bar_id, NT);
            load<S - 1, S - 1>(x, buf, t);
            if (xp.stride == 0) team_sync(bar_id, NT);
            buf = xp.next();
            store<S, S - 1>(y, buf, t);
            team_sync(bar_id, NT);
            load<S - 1, S - 1>(y, buf, t);
            if (xp.stride == 0) team_sync(bar_id, NT);
            inverse_two_from<S - 1>(x, y, xp, tw2, t, bar_id);
        }
    }
    __device__ static __forceinline__ void inverse_two(cpair *x, cpair *y, ExchPair &xp, const float4 *tw2, int t,
                                                       int bar_id) {
        inverse_two_from<NS - 1>(x, y, xp, tw2, t, bar_id);
        fold_consts<true>(x);
        fold_consts<true>(y);
    }
};

}  // namespace tfheb
