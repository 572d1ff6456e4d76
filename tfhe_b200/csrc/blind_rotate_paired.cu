// blind_rotate_paired.cu -- the split-FP32 blind rotation with two transforms per thread and the
// digit spectra in tensor memory (tfhe_blindRotate_FFT, lwe-bootstrapping-functions-fft.cpp:88-112,
// with the external product tGswFFTExternMulToTLwe, tgsw-fft-operations.cpp:89-114).
//
// The same work, in the same order per accumulator, as blind_rotate_kernel<float, ..., SPLIT>, so
// both give the same bits.  The schedule differs:
//   * The gadget digits of a step are transformed two at a time on packed f32x2 (TeamFft2: one
//     packed instruction performs the same scalar operation on both transforms), and each output
//     polynomial's two key limbs are inverted together: half the FP32 instructions of the
//     transforms, and one 16-byte exchange access per point of two transforms.
//   * The (k+1)l digit spectra of a step are parked in tensor memory (TMEM, 256 KB per SM, which the
//     path otherwise leaves idle), one 32-lane row per thread.  The multiply-accumulate then runs one
//     output polynomial at a time, so two limb accumulators (32 registers) are live instead of
//     2(k+1) (64 registers at k = 1), and the 128 registers of 15 warps per SM hold the paired
//     transforms without spilling.
//   * The key ring holds half rows, one output polynomial's slots of one digit row (8 KB at N =
//     1024), streamed in the order of the multiply-accumulate: per step, output 0 over the digits,
//     then output 1.
//   * XT: the step's rotated words (32 per thread) wait in TMEM, in columns the spectra leave free,
//     between the rotation and the digit extraction, so they hold no registers across the forward
//     transforms.  IL (with XT): 1 transforms the first two digit pairs together, stage by stage
//     (TeamFft2::forward_two: independent chains, one twiddle load for both); 2 also runs both
//     outputs' multiply-accumulates first and their inverse pairs together (inverse_two); 3 as 2,
//     with output 0's inverse input waiting in the rotated words' columns during output 1's
//     multiply-accumulate; 7 as 3, with the keys of slot pairs 0 and 1 of digit d + 1 loaded during
//     digit d's multiply-accumulate (16 registers of look-ahead).  Every accumulator and transform
//     still sees the same operations in the same order, so all variants give the same bits.
// Every mbarrier wait is bounded as in blind_rotate_kernel.  Warp 0 allocates the TMEM columns at
// the start and frees them after every consumer thread has passed a final barrier, on every path
// (a wait that runs out only makes the remaining waits return at once).
#include <cuda_runtime.h>
#include <stdint.h>

#include "async_copy.cuh"
#include "br_common.cuh"
#include "fft.cuh"
#include "internal.h"
#include "tmem.cuh"

namespace tfheb {

namespace {

// Two digits as floats in one packed pair: the bits of 1.5*2^23 + d of each (digit mask and OR in one
// logic op), then one packed subtraction of the bias.  sub_bias_neg gives -(x - bias) as bias - x, the
// same value (round to nearest is symmetric; only the sign of a zero may differ, which no later
// operation can turn into a different rounded result).
__device__ __forceinline__ float2 digit_pair(uint32_t a, uint32_t b) {
    return make_float2(__int_as_float(0x4B400000u | a), __int_as_float(0x4B400000u | b));
}

}  // namespace

// ---- shared memory and TMEM budget ---------------------------------------------------------------

template <int N, int L, int G, int D, int XB, bool PW = true, bool XT = false>
struct PairLayout {
    static constexpr int M = N / 2, NT = M / kR, KP1 = 2, KPL = KP1 * L;
    static constexpr uint32_t half = (uint32_t)M * 16;  // one output's slots of one key row
    static constexpr size_t bars = 0;                   // full[D], empty[D], abort flag, TMEM address
    static constexpr size_t ring = (2 * D * 8 + 8 + 127) / 128 * 128;
    static constexpr size_t tables = ring + (size_t)D * half;
    static constexpr size_t tables_bytes = 16 * (size_t)tw_offset<M>(FftPlan<M>::NS);
    static constexpr size_t teams = tables + tables_bytes;
    static constexpr size_t team_acc = 4 * (size_t)KP1 * N;
    static constexpr size_t team_xbuf = 16 * (size_t)Exch<double, M>::slots;
    static constexpr size_t team_bytes = team_acc + XB * team_xbuf;
    static constexpr size_t bytes = teams + G * team_bytes;
    static constexpr int threads = G * NT + (PW ? 32 : 0);
    // TMEM: KPL spectra of 16 words per thread; warps of one lane quadrant take column slots in turn
    static constexpr int warps = G * NT / 32;
    static constexpr int cols_per_warp = KPL * 16;
    static constexpr int spectra_cols = (warps + 3) / 4 * cols_per_warp;
    // XT: the step's rotated words (32 per thread) wait in TMEM during the forward transforms
    static constexpr int xr_col = spectra_cols;
    static constexpr int cols_needed = spectra_cols + (XT ? (warps + 3) / 4 * 32 : 0);
    static constexpr int tmem_cols = cols_needed <= 32 ? 32 : cols_needed <= 64 ? 64 : cols_needed <= 128 ? 128
                                   : cols_needed <= 256 ? 256 : 512;
    static_assert(cols_needed <= 512, "TMEM columns of the variant");
    static_assert(bytes <= 227 * 1024, "shared memory of the variant");
    static_assert(NT % 32 == 0, "whole warps per team");
    static_assert(half % 16 == 0, "bulk copies need 16-byte sizes");
};

// PW: a key-streaming warp issues the half-row copies.  Without it, thread 0 issues them, as in
// blind_rotate_kernel: the first D at the start, then each one as soon as every team has released its
// slot, tested after each of its own half rows and waited for only when thread 0 needs one not yet
// issued.  That frees the producer warp's registers (N = 2048 with two teams: 8 warps, 255 registers).
template <int N, int L, int G, int D, int XB, bool PW, bool XT, int IL>
__global__ void __launch_bounds__(G *(N / 16) + (PW ? 32 : 0), 1) blind_rotate_paired_kernel(const BrArgs args) {
    using Lay = PairLayout<N, L, G, D, XB, PW, XT>;
    constexpr int M = N / 2, NT = M / kR, KP1 = 2, KPL = KP1 * L;
    using F2 = TeamFft2<M>;
    extern __shared__ __align__(128) unsigned char smem[];

    const int tid = threadIdx.x, warp = tid >> 5;
    const int consumers = G * NT;
    const int active_teams = min(G, args.boots - (int)blockIdx.x * G);
    const uint32_t bar0 = smem_addr(smem + Lay::bars);
    auto full_bar = [&](int s) { return bar0 + 8u * s; };
    auto empty_bar = [&](int s) { return bar0 + 8u * (D + s); };
    volatile int32_t *abort_flag = reinterpret_cast<volatile int32_t *>(smem + Lay::bars + 16 * D);
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + Lay::bars + 16 * D + 4);
    const uint32_t ring = smem_addr(smem + Lay::ring);

    if (tid == 0) {
        for (int s = 0; s < D; s++) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), (uint32_t)(active_teams * NT));
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncwarp();  // the allocation is a warp-wide instruction: warp 0 converged after thread 0's branch
    if (warp == 0) tmem_alloc(smem_addr(tmem_slot), Lay::tmem_cols);
    {
        const int4 *g_tab = reinterpret_cast<const int4 *>(args.tables2);
        int4 *s_tab4 = reinterpret_cast<int4 *>(smem + Lay::tables);
        for (int i = tid; i < (int)(Lay::tables_bytes / 16); i += blockDim.x) s_tab4[i] = g_tab[i];
    }
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;

    // half rows in consumption order: per step, output v = 0 then 1, each over the digits d
    const int total_chunks = args.nsteps * KP1 * KPL;
    auto issue_row = [&](int c) {
        const int s = c % D;
        const int step = c / (KP1 * KPL), rem = c - step * (KP1 * KPL);
        const int v = rem / KPL, d = rem - v * KPL;
        const size_t src = ((size_t)(step * KPL + d) * KP1 + v) * Lay::half;
        mbar_arrive_expect_tx(full_bar(s), Lay::half);
        bulk_copy_g2s(ring + (uint32_t)s * Lay::half, args.bsk + src, Lay::half, full_bar(s));
    };
    int issued = 0;  // !PW: half rows issued by thread 0
    bool issuing = !PW && tid == 0 && !args.stall_producer;
    if (issuing)
        for (; issued < min(D, total_chunks); issued++) issue_row(issued);

    // ---------------- producer warp: stream the key half rows ----------------
    if (tid >= consumers) {
        if (tid == consumers) {
            int sent = 0;
            if (!args.stall_producer) {
                for (int c = 0; c < total_chunks; c++) {
                    const int s = c % D;
                    if (c >= D && !wait_bounded(empty_bar(s), ((c / D) - 1) & 1, abort_flag, args.timeout_ns, args.err))
                        break;
                    issue_row(c);
                    sent = c + 1;
                }
            }
            volatile int32_t no_abort = 0;
            for (int c = (sent > D ? sent - D : 0); c < sent; c++)
                wait_bounded(full_bar(c % D), (c / D) & 1, &no_abort, args.timeout_ns, args.err);
        }
        return;
    }

    // ---------------- consumer teams ----------------
    const int team = tid / NT;
    const int t = tid - team * NT;
    if (team >= active_teams) return;  // no TMEM use, not counted in any barrier below
    const int boot = blockIdx.x * G + team;
    const int bar_id = 1 + team;
    constexpr int kAllBar = 15;
    static_assert(G < kAllBar, "named barrier ids");

    unsigned char *tb = smem + Lay::teams + (size_t)team * Lay::team_bytes;
    uint32_t *s_acc = reinterpret_cast<uint32_t *>(tb);
    ExchPair xp{tb + Lay::team_acc, XB == 2 ? (uint32_t)Lay::team_xbuf : 0u, 0u};
    const float4 *s_tw2 = reinterpret_cast<const float4 *>(smem + Lay::tables);
    // this thread's TMEM row: lane quadrant of its warp, the warp's column slot within the quadrant
    const uint32_t tmem_row = tmem_base + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)((warp >> 2) * Lay::cols_per_warp);
    const uint32_t tmem_xr = tmem_base + ((uint32_t)((warp & 3) * 32) << 16) + (uint32_t)(Lay::xr_col + (warp >> 2) * 32);

    const int32_t *my_bara = args.bara + (size_t)boot * args.bara_stride;
    if (args.acc_in) {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(args.acc_in) + (size_t)boot * KP1 * N;
        for (int i = t; i < KP1 * N; i += NT) s_acc[i] = src[i];
    } else {
        // acc = (0, X^{2N-barb} * [mu,...,mu])  (lwe-bootstrapping-functions-fft.cpp:142-145)
        const int e = 2 * N - my_bara[args.nsteps];
        for (int i = t; i < N; i += NT) s_acc[i] = 0u;
        for (int j = t; j < N; j += NT) {
            int src = j - e;
            uint32_t neg = 0;
            while (src < 0) {
                src += N;
                neg ^= 1u;
            }
            s_acc[N + j] = neg ? 0u - (uint32_t)args.mu : (uint32_t)args.mu;
        }
    }
    team_sync(bar_id, NT);

    // gadget constants (tgsw.cpp:7-29)
    const int Bgbit = args.Bgbit;
    uint32_t offset = 0;
#pragma unroll
    for (int q = 0; q < L; q++) offset += 1u << (32 - (q + 1) * Bgbit);
    offset *= 1u << (Bgbit - 1);
    const uint32_t maskBg = (1u << Bgbit) - 1u;
    const float digit_bias = 12582912.0f + float(1 << (Bgbit - 1));

    int a_next = args.nsteps > 0 ? my_bara[0] : 0;  // rotation amounts, loaded one step ahead
    for (int step = 0; step < args.nsteps; step++) {
        const int ai = a_next & (2 * N - 1);
        if (step + 1 < args.nsteps) a_next = my_bara[step + 1];

        // 1. (X^a - 1) * poly + offset of both polynomials, words j = t + NT r and j + M
        uint32_t xr[KP1][2 * kR];
#pragma unroll
        for (int u = 0; u < KP1; u++)
#pragma unroll
            for (int r = 0; r < kR; r++) {
                const int j = t + NT * r;
                xr[u][r] = rot_minus_one<N>(s_acc + u * N, j, ai) + offset;
                xr[u][kR + r] = rot_minus_one<N>(s_acc + u * N, j + M, ai) + offset;
            }
        if constexpr (XT) {
            tmem_st32(tmem_xr, reinterpret_cast<uint32_t(&)[32]>(xr));
            tmem_wait_st();
        }
        // 2. digits two at a time in chain order d = u*L + q, forward transforms, spectra to TMEM
        const float2 bias2 = make_float2(digit_bias, digit_bias);
        // digit polynomials d0 (words xa) and d0 + 1 (words xb) as one packed pair: a_j - i a_{j+M}
        // of each (the twist is folded into the FFT)
        auto digits = [&](cpair(&z)[kR], int d0, const uint32_t(&xa)[2 * kR], const uint32_t(&xb)[2 * kR]) {
            const int sh0 = 32 - (d0 % L + 1) * Bgbit, sh1 = 32 - ((d0 + 1) % L + 1) * Bgbit;
#pragma unroll
            for (int r = 0; r < kR; r++) {
                const float2 lo = digit_pair((xa[r] >> sh0) & maskBg, (xb[r] >> sh1) & maskBg);
                const float2 hi = digit_pair((xa[kR + r] >> sh0) & maskBg, (xb[kR + r] >> sh1) & maskBg);
                z[r] = {sub2(lo, bias2), sub2(bias2, hi)};
            }
        };
        // spectrum words in multiply-accumulate order: per register pair m, re(2m), re(2m+1), im(2m),
        // im(2m+1); digit d0 then digit d0 + 1
        auto park = [&](const cpair(&z)[kR], int d0) {
            uint32_t w[32];
#pragma unroll
            for (int m = 0; m < kR / 2; m++) {
                w[4 * m + 0] = __float_as_uint(z[2 * m].re.x);
                w[4 * m + 1] = __float_as_uint(z[2 * m + 1].re.x);
                w[4 * m + 2] = __float_as_uint(z[2 * m].im.x);
                w[4 * m + 3] = __float_as_uint(z[2 * m + 1].im.x);
                w[16 + 4 * m + 0] = __float_as_uint(z[2 * m].re.y);
                w[16 + 4 * m + 1] = __float_as_uint(z[2 * m + 1].re.y);
                w[16 + 4 * m + 2] = __float_as_uint(z[2 * m].im.y);
                w[16 + 4 * m + 3] = __float_as_uint(z[2 * m + 1].im.y);
            }
            tmem_st32(tmem_row + (uint32_t)(d0 * 16), w);
        };
        if constexpr (IL >= 1) {
            // pairs (0, 1) and (2, 3) transformed together, then (4, 5)
            static_assert(XT && L == 3 && KP1 == 2, "interleaved pairs: k = 1, l = 3, words in TMEM");
            uint32_t xw[KP1][2 * kR];
            tmem_ld16(tmem_xr, xw[0]);
            tmem_ld16(tmem_xr + 16u, xw[1]);
            tmem_wait_ld16(xw[0]);
            tmem_wait_ld16(xw[1]);
            cpair z0[kR], z1[kR];
            digits(z0, 0, xw[0], xw[0]);
            digits(z1, 2, xw[0], xw[1]);
            F2::forward_two(z0, z1, xp, s_tw2, t, bar_id);
            park(z0, 0);
            park(z1, 2);
            tmem_ld16(tmem_xr + 16u, xw[1]);
            tmem_wait_ld16(xw[1]);
            cpair z2[kR];
            digits(z2, 4, xw[1], xw[1]);
            F2::forward(z2, xp, s_tw2, t, bar_id);
            park(z2, 4);
        } else {
#pragma unroll
            for (int d0 = 0; d0 < KPL; d0 += 2) {
                const int u0 = d0 / L, u1 = (d0 + 1) / L;
                uint32_t xw[KP1][2 * kR];  // XT: the words of the polynomials this pair reads, from TMEM
                if constexpr (XT) {
                    tmem_ld16(tmem_xr + (uint32_t)(16 * u0), xw[u0]);
                    if (u1 != u0) tmem_ld16(tmem_xr + (uint32_t)(16 * u1), xw[u1]);
                    tmem_wait_ld16(xw[u0]);
                    if (u1 != u0) tmem_wait_ld16(xw[u1]);
                }
                cpair z[kR];
                digits(z, d0, XT ? xw[u0] : xr[u0], XT ? xw[u1] : xr[u1]);
                F2::forward(z, xp, s_tw2, t, bar_id);
                park(z, d0);
            }
        }
        tmem_wait_st();

        // 3. per output polynomial: multiply-accumulate over the digits against the key half rows,
        //    then both limbs' inverse transforms together, exact rounding, accumulate
        auto mac = [&](int v, cpair(&ah)[kR / 2], cpair(&al)[kR / 2]) {
#pragma unroll
            for (int m = 0; m < kR / 2; m++) {
                ah[m] = {{0.f, 0.f}, {0.f, 0.f}};
                al[m] = {{0.f, 0.f}, {0.f, 0.f}};
            }
            if constexpr (IL == 7) {
                // the keys of the first PF slot pairs of digit d + 1 load during digit d's arithmetic
                static_assert(PW, "IL = 7 needs the producer warp");
                constexpr int PF = 2;  // slot pairs (2 float4 each) ahead; 3 or 4 measured no faster
                const int c0 = (step * KP1 + v) * KPL;
                auto slot = [&](int c) {
                    return reinterpret_cast<const float4 *>(smem + Lay::ring + (size_t)(c % D) * Lay::half) + t;
                };
                auto mac_m = [&](int m, const uint32_t(&f)[16], float4 kh, float4 kl) {
                    const cpair zp{make_float2(__uint_as_float(f[4 * m]), __uint_as_float(f[4 * m + 1])),
                                   make_float2(__uint_as_float(f[4 * m + 2]), __uint_as_float(f[4 * m + 3]))};
                    const float2 nzi = mul2(zp.im, make_float2(-1.f, -1.f));
                    cmac_pair(ah[m], zp, nzi, kh);
                    cmac_pair(al[m], zp, nzi, kl);
                };
                uint32_t fb[2][16];
                tmem_ld16(tmem_row, fb[0]);
                wait_bounded(full_bar(c0 % D), (c0 / D) & 1, abort_flag, args.timeout_ns, args.err);
                float4 kn[2 * PF];
                {
                    const float4 *kp = slot(c0);
#pragma unroll
                    for (int e = 0; e < 2 * PF; e++) kn[e] = kp[e * NT];
                }
                tmem_wait_ld16(fb[0]);
#pragma unroll
                for (int d = 0; d < KPL; d++) {
                    const int c = c0 + d;
                    const float4 *kp = slot(c);
                    uint32_t(&f)[16] = fb[d & 1];
                    if (d + 1 < KPL) tmem_ld16(tmem_row + (uint32_t)((d + 1) * 16), fb[(d + 1) & 1]);
                    float4 kc[kR];  // this digit's keys: the first 2 PF from the look-ahead
#pragma unroll
                    for (int e = 0; e < 2 * PF; e++) kc[e] = kn[e];
#pragma unroll
                    for (int e = 2 * PF; e < kR; e++) kc[e] = kp[e * NT];
                    if (d + 1 < KPL) {
                        wait_bounded(full_bar((c + 1) % D), ((c + 1) / D) & 1, abort_flag, args.timeout_ns, args.err);
                        const float4 *kq = slot(c + 1);
#pragma unroll
                        for (int e = 0; e < 2 * PF; e++) kn[e] = kq[e * NT];
                    }
#pragma unroll
                    for (int m = 0; m < kR / 2; m++) mac_m(m, f, kc[2 * m], kc[2 * m + 1]);
                    mbar_arrive(empty_bar(c % D));
                    if (d + 1 < KPL) tmem_wait_ld16(fb[(d + 1) & 1]);
                }
                return;
            }
            // digit spectra from TMEM, the next one loading while this one is multiplied
            uint32_t fb[2][16];
            tmem_ld16(tmem_row, fb[0]);
            tmem_wait_ld16(fb[0]);
#pragma unroll
            for (int d = 0; d < KPL; d++) {
                const int c = (step * KP1 + v) * KPL + d, s = c % D;
                uint32_t(&f)[16] = fb[d & 1];
                if (d + 1 < KPL) tmem_ld16(tmem_row + (uint32_t)((d + 1) * 16), fb[(d + 1) & 1]);
                if constexpr (!PW) {
                    // thread 0 issues every half row before anyone waits for it
                    while (issuing && issued <= c && issued < total_chunks) {
                        if (!wait_bounded(empty_bar(issued % D), ((issued / D) - 1) & 1, abort_flag, args.timeout_ns,
                                          args.err)) {
                            issuing = false;
                            break;
                        }
                        issue_row(issued++);
                    }
                }
                wait_bounded(full_bar(s), (c / D) & 1, abort_flag, args.timeout_ns, args.err);
                // half row: [m][limb][t] x float4 {re(2m), re(2m+1), im(2m), im(2m+1)}
                const float4 *kp = reinterpret_cast<const float4 *>(smem + Lay::ring + (size_t)s * Lay::half) + t;
#pragma unroll
                for (int m = 0; m < kR / 2; m++) {
                    const cpair zp{make_float2(__uint_as_float(f[4 * m]), __uint_as_float(f[4 * m + 1])),
                                   make_float2(__uint_as_float(f[4 * m + 2]), __uint_as_float(f[4 * m + 3]))};
                    const float2 nzi = mul2(zp.im, make_float2(-1.f, -1.f));
                    cmac_pair(ah[m], zp, nzi, kp[(2 * m) * NT]);
                    cmac_pair(al[m], zp, nzi, kp[(2 * m + 1) * NT]);
                }
                mbar_arrive(empty_bar(s));
                if constexpr (!PW) {
                    while (issuing && issued < total_chunks &&
                           mbar_test_wait(empty_bar(issued % D), ((issued / D) - 1) & 1))
                        issue_row(issued++);
                }
                if (d + 1 < KPL) tmem_wait_ld16(fb[(d + 1) & 1]);
            }
        };
        // (hi, lo) per slot for the paired inverse
        auto limbs = [&](cpair(&x)[kR], const cpair(&ah)[kR / 2], const cpair(&al)[kR / 2]) {
#pragma unroll
            for (int m = 0; m < kR / 2; m++) {
                x[2 * m] = {make_float2(ah[m].re.x, al[m].re.x), make_float2(ah[m].im.x, al[m].im.x)};
                x[2 * m + 1] = {make_float2(ah[m].re.y, al[m].re.y), make_float2(ah[m].im.y, al[m].im.y)};
            }
        };
        auto accumulate = [&](int v, const cpair(&x)[kR]) {
            uint32_t *poly = s_acc + v * N;
#pragma unroll
            for (int r = 0; r < kR; r++) {  // (c_j - i c_{j+M}) of each limb, the high limb weighted 2^S
                const int j = t + NT * r;
                poly[j] += (round_f32_mod32(x[r].re.x) << args.split_shift) + (uint32_t)__float2ll_rn(x[r].re.y);
                poly[j + M] += (round_f32_mod32(-x[r].im.x) << args.split_shift) + (uint32_t)__float2ll_rn(-x[r].im.y);
            }
        };
        if constexpr (IL == 3 || IL == 7) {
            // output 0's inverse input waits in the rotated words' TMEM columns (free after the
            // forward transforms) during output 1's multiply-accumulate; then both inverse pairs
            // interleaved
            cpair x0[kR], x1[kR];
            {
                cpair ah[kR / 2], al[kR / 2];
                mac(0, ah, al);
                limbs(x0, ah, al);
            }
            tmem_st32(tmem_xr, reinterpret_cast<uint32_t(&)[32]>(x0));
            {
                cpair ah[kR / 2], al[kR / 2];
                mac(1, ah, al);
                limbs(x1, ah, al);
            }
            tmem_wait_st();
            tmem_ld16(tmem_xr, reinterpret_cast<uint32_t(&)[16]>(x0[0]));
            tmem_ld16(tmem_xr + 16u, reinterpret_cast<uint32_t(&)[16]>(x0[kR / 2]));
            tmem_wait_ld16(reinterpret_cast<uint32_t(&)[16]>(x0[0]));
            tmem_wait_ld16(reinterpret_cast<uint32_t(&)[16]>(x0[kR / 2]));
            F2::inverse_two(x0, x1, xp, s_tw2, t, bar_id);
            accumulate(0, x0);
            accumulate(1, x1);
        } else if constexpr (IL == 2) {
            // both outputs' accumulators, then both inverse pairs interleaved
            cpair ah0[kR / 2], al0[kR / 2], ah1[kR / 2], al1[kR / 2];
            mac(0, ah0, al0);
            mac(1, ah1, al1);
            cpair x0[kR], x1[kR];
            limbs(x0, ah0, al0);
            limbs(x1, ah1, al1);
            F2::inverse_two(x0, x1, xp, s_tw2, t, bar_id);
            accumulate(0, x0);
            accumulate(1, x1);
        } else {
#pragma unroll 1
            for (int v = 0; v < KP1; v++) {
                cpair ah[kR / 2], al[kR / 2];
                mac(v, ah, al);
                cpair x[kR];
                limbs(x, ah, al);
                F2::inverse(x, xp, s_tw2, t, bar_id);
                accumulate(v, x);
            }
        }
        team_sync(bar_id, NT);
    }

    uint32_t *dst = reinterpret_cast<uint32_t *>(args.acc_out) + (size_t)boot * KP1 * N;
    for (int i = t; i < KP1 * N; i += NT) dst[i] = s_acc[i];
    if constexpr (!PW) {
        // after an abort, drain the copies still in flight before the CTA may exit (bounded waits)
        if (tid == 0) {
            volatile int32_t no_abort = 0;
            for (int r = (issued > D ? issued - D : 0); r < issued; r++)
                wait_bounded(full_bar(r % D), (r / D) & 1, &no_abort, args.timeout_ns, args.err);
        }
    }

    // every consumer's TMEM accesses are complete (each load waited; stores waited per step)
    tmem_fence_before_sync();
    team_sync(kAllBar, active_teams * NT);
    tmem_fence_after_sync();
    __syncwarp();
    if (warp == 0) tmem_free(tmem_base, Lay::tmem_cols);
}

template <int N, int L, int G, int D, int XB, bool PW, bool XT, int IL = 0>
static cudaError_t launch_paired_impl(const BrArgs &a, cudaStream_t s) {
    using Lay = PairLayout<N, L, G, D, XB, PW, XT>;
    if (!a.tables2) return cudaErrorInvalidValue;
    auto kern = blind_rotate_paired_kernel<N, L, G, D, XB, PW, XT, IL>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::bytes);
    if (e != cudaSuccess) return e;
    const int grid = (a.boots + G - 1) / G;
    kern<<<grid, Lay::threads, Lay::bytes, s>>>(a);
    return cudaGetLastError();
}

template <int N, int L, int G, int D, int XB, bool PW>
cudaError_t launch_paired(const BrArgs &a, cudaStream_t s) {
    return launch_paired_impl<N, L, G, D, XB, PW, false>(a, s);
}
template <int N, int L, int G, int D, int XB>
cudaError_t launch_paired_il(const BrArgs &a, cudaStream_t s) {
    return launch_paired_impl<N, L, G, D, XB, true, true, 1>(a, s);
}
template <int N, int L, int G, int D, int XB>
cudaError_t launch_paired_il2(const BrArgs &a, cudaStream_t s) {
    return launch_paired_impl<N, L, G, D, XB, true, true, 2>(a, s);
}
template <int N, int L, int G, int D, int XB>
cudaError_t launch_paired_il3(const BrArgs &a, cudaStream_t s) {
    return launch_paired_impl<N, L, G, D, XB, true, true, 3>(a, s);
}
template <int N, int L, int G, int D, int XB>
cudaError_t launch_paired_il7(const BrArgs &a, cudaStream_t s) {
    return launch_paired_impl<N, L, G, D, XB, true, true, 7>(a, s);
}


template cudaError_t launch_paired<1024, 3, 7, 8, 1, true>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired<1024, 3, 7, 12, 1, true>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired<1024, 3, 7, 4, 2, true>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired<1024, 3, 6, 6, 2, true>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired<2048, 3, 2, 4, 2, false>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired<2048, 3, 2, 4, 2, true>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired<2048, 3, 3, 4, 1, true>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired_il<1024, 3, 7, 12, 1>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired_il<2048, 3, 3, 6, 1>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired_il2<1024, 3, 7, 12, 1>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired_il2<2048, 3, 3, 6, 1>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired_il3<1024, 3, 7, 12, 1>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired_il3<2048, 3, 3, 6, 1>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired_il7<1024, 3, 7, 12, 1>(const BrArgs &, cudaStream_t);


template cudaError_t launch_paired_il3<1024, 3, 6, 12, 1>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired_il3<1024, 3, 5, 12, 1>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired_il3<1024, 3, 4, 12, 1>(const BrArgs &, cudaStream_t);
template cudaError_t launch_paired_il3<1024, 3, 3, 12, 1>(const BrArgs &, cudaStream_t);

}  // namespace tfheb
