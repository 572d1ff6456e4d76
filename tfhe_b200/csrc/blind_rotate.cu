// blind_rotate.cu -- persistent blind rotation on sm_100a (tfhe_blindRotate_FFT,
// lwe-bootstrapping-functions-fft.cpp:88-112, with tfhe_MuxRotate_FFT :67-76 and the external
// product tGswFFTExternMulToTLwe, tgsw-fft-operations.cpp:89-114).
//
// One CTA = G "teams" (one bootstrap each, N/16 threads per team) + one producer warp.
//   * Each team keeps its accumulator TLWE (k+1 polynomials of N Torus32) in shared memory for all
//     n CMUX steps.  Per step: rotation (X^a - 1)*acc, gadget decomposition, a forward negacyclic FFT
//     per digit polynomial (fft.cuh), multiply-accumulate against the bootstrapping-key row in the
//     FFT domain, inverse FFTs, rounding back to Torus32 and accumulation.
//   * The bootstrapping key is streamed once per CTA: the producer warp copies each key row
//     ((k+1) x N/2 slots x 16 bytes = 16 KB at N=1024) with a bulk asynchronous copy (TMA engine,
//     cp.async.bulk, no multicast) into a D-stage shared-memory ring guarded by mbarriers; all G teams
//     read the same stage.  L2->SM key traffic is therefore 62 MB per G bootstraps instead of per
//     bootstrap.
//   * Every mbarrier wait is bounded (%globaltimer).  On expiry the CTA raises a shared abort flag,
//     every later wait returns at once (the FFT barriers stay uniform, so nothing hangs), the
//     producer drains its in-flight copies, and the host reads TFHEB_ERR_TIMEOUT from the error word.
//
// Precision forms:
//   FP64  (SPLIT=false): key row slot = double2 B_k / M; products rounded with the 1.5*2^52 addition
//          (exact round-to-nearest for |x| < 2^51), reduced mod 2^32.
//   split (SPLIT=true):  key coefficient c = hi * 2^S + lo (S from default_split_shift); per register
//          pair (2m, 2m+1) and limb, float4 {re(2m), re(2m+1), im(2m), im(2m+1)} / M, one 16-byte load
//          per packed multiply-accumulate.  The high-limb product sums round to their exact integers
//          (S keeps their FP32 error far below 1/2); the low-limb sums round to the nearest integer of
//          their FP32 value; the two recombine as hi * 2^S + lo mod 2^32.
#include <cuda_runtime.h>
#include <stdint.h>

#include "async_copy.cuh"
#include "br_common.cuh"
#include "fft.cuh"
#include "internal.h"

namespace tfheb {

// ---- shared-memory layout ---------------------------------------------------------------------

template <typename T, int N, int K, int G, int D, bool PW = true>
struct BrLayout {
    static constexpr int M = N / 2, NT = M / kR, KP1 = K + 1;
    static constexpr uint32_t chunk = (uint32_t)KP1 * M * 16;  // one key row (step, p): all v, all slots
    static constexpr size_t bars = 0;                           // full[D], empty[D], abort flag
    static constexpr size_t ring = (2 * D * 8 + 4 + 127) / 128 * 128;  // the barrier block, then the ring
    static constexpr size_t tables = ring + (size_t)D * chunk;
    static constexpr size_t tables_bytes = tw_table_bytes<T, M>();
    static constexpr size_t teams = tables + tables_bytes;
    static constexpr size_t team_acc = 4 * (size_t)KP1 * N;
    static constexpr size_t team_xbuf = ((size_t)Exch<T, M>::bytes + 15) / 16 * 16;  // one exchange buffer
    // two alternating exchange buffers: one barrier per exchange (at N = 2048 with the per-exchange
    // float2 maps: 69.5 ms per 2048 split bootstraps against 69.7-70.5 ms with one buffer)
    static constexpr int xbufs = 2;
    static constexpr size_t team_buf = xbufs * team_xbuf;
    // the rotated accumulator polynomial being decomposed (N words), read once per digit: kept in a
    // per-team shared scratch when registers are tight (more than 256 threads per CTA, so at most 168
    // registers each) and the scratch fits beside the key ring, else in registers.  A deeper ring
    // measured faster than the scratch (36.15 ms per 4096 split bootstraps at G = 7, D = 6 without it,
    // 36.6 ms at D = 4 with it), and a lone team with 255 registers runs slower with it.
    static constexpr size_t kMaxSmem = 227 * 1024;
    static constexpr int threads = G * (N / 16) + (PW ? 32 : 0);
    static constexpr bool rot_in_smem =
        threads > 256 && teams + G * (team_acc + team_buf + 4 * (size_t)N) <= kMaxSmem;
    static constexpr size_t team_rot = rot_in_smem ? 4 * (size_t)N : 0;
    __host__ __device__ static size_t team_bytes(int) { return team_acc + team_buf + team_rot; }
    __host__ __device__ static size_t bytes(int nsteps) { return teams + G * team_bytes(nsteps); }
    static_assert(2 * D * 8 + 4 <= ring, "barrier block");
    static_assert(teams + G * (team_acc + team_buf) <= kMaxSmem, "shared memory of the variant");
};



// PW: a key-streaming warp issues the row copies.  Without it (G teams only), thread 0 issues them:
// the first D at the start, then each row as soon as every team has released its slot, tested after
// each of its own rows and waited for only when thread 0 needs a row not yet issued.  That frees the
// producer warp's registers: 4 FP64 teams are 256 threads, which may use 255 registers each.
// EXT: the external product alone (tGswExternProduct, tgsw-functions.cpp:416-431): each step computes
// acc = bk_step (x) acc, without the rotation (X^a - 1) and without adding the old accumulator; the
// rotation amounts are not read.  Only a few one-bootstrap-per-CTA variants are compiled with it.
template <typename T, int N, int K, int L, bool SPLIT, int G, int D, bool PW = true, bool EXT = false>
__global__ void __launch_bounds__(G *(N / 16) + (PW ? 32 : 0), 1) blind_rotate_kernel(const BrArgs args) {
    using Lay = BrLayout<T, N, K, G, D, PW>;
    constexpr int M = N / 2, NT = M / kR, KP1 = K + 1, KPL = KP1 * L;
    using F = TeamFft<T, M, kR>;
    extern __shared__ __align__(128) unsigned char smem[];

    const int tid = threadIdx.x;
    const int consumers = G * NT;
    const int active_teams = min(G, args.boots - (int)blockIdx.x * G);
    const uint32_t bar0 = smem_addr(smem + Lay::bars);
    auto full_bar = [&](int s) { return bar0 + 8u * s; };
    auto empty_bar = [&](int s) { return bar0 + 8u * (D + s); };
    volatile int32_t *abort_flag = reinterpret_cast<volatile int32_t *>(smem + Lay::bars + 16 * D);
    const uint32_t ring = smem_addr(smem + Lay::ring);

    if (tid == 0) {
        for (int s = 0; s < D; s++) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), (uint32_t)(active_teams * NT));
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    cplx<T> *s_tab = reinterpret_cast<cplx<T> *>(smem + Lay::tables);
    {
        const int4 *g_tab = reinterpret_cast<const int4 *>(args.tables);
        int4 *s_tab4 = reinterpret_cast<int4 *>(smem + Lay::tables);
        for (int i = tid; i < (int)(Lay::tables_bytes / 16); i += blockDim.x) s_tab4[i] = g_tab[i];
    }
    __syncthreads();

    const int total_chunks = args.nsteps * KPL;
    // row c into its ring slot (the slot's previous row released by every team)
    auto issue_row = [&](int c) {
        const int s = c % D;
        mbar_arrive_expect_tx(full_bar(s), Lay::chunk);
        bulk_copy_g2s(ring + (uint32_t)s * Lay::chunk, args.bsk + (size_t)c * Lay::chunk, Lay::chunk, full_bar(s));
    };
    int issued = 0;        // !PW: rows issued by thread 0
    bool issuing = !PW && tid == 0 && !args.stall_producer;
    if (issuing)
        for (; issued < min(D, total_chunks); issued++) issue_row(issued);

    // ---------------- producer warp: stream the key rows ----------------
    if (tid >= consumers) {
        if (tid == consumers) {
            int sent = 0;
            if (!args.stall_producer) {
                for (int c = 0; c < total_chunks; c++) {
                    const int s = c % D;
                    if (c >= D && !wait_bounded(empty_bar(s), ((c / D) - 1) & 1, abort_flag, args.timeout_ns, args.err))
                        break;
                    mbar_arrive_expect_tx(full_bar(s), Lay::chunk);
                    bulk_copy_g2s(ring + (uint32_t)s * Lay::chunk, args.bsk + (size_t)c * Lay::chunk, Lay::chunk,
                                  full_bar(s));
                    sent = c + 1;
                }
            }
            // drain the copies still in flight before the CTA may exit (each wait bounded)
            volatile int32_t no_abort = 0;
            for (int c = (sent > D ? sent - D : 0); c < sent; c++)
                wait_bounded(full_bar(c % D), (c / D) & 1, &no_abort, args.timeout_ns, args.err);
        }
        return;
    }

    // ---------------- consumer teams ----------------
    const int team = tid / NT;
    const int t = tid - team * NT;
    if (team >= active_teams) return;  // not counted in the empty barriers; no CTA barrier follows
    const int boot = blockIdx.x * G + team;
    const int bar_id = 1 + team;

    unsigned char *tb = smem + Lay::teams + (size_t)team * Lay::team_bytes(args.nsteps);
    uint32_t *s_acc = reinterpret_cast<uint32_t *>(tb);
    ExchPair xp{tb + Lay::team_acc, Lay::xbufs == 2 ? (uint32_t)Lay::team_xbuf : 0u, 0u};
    uint32_t *s_rot = reinterpret_cast<uint32_t *>(tb + Lay::team_acc + Lay::team_buf);
    const cplx<T> *s_tw = s_tab;

    const int32_t *my_bara = EXT ? nullptr : args.bara + (size_t)boot * args.bara_stride;
    if (EXT || args.acc_in) {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(args.acc_in) + (size_t)boot * KP1 * N;
        for (int i = t; i < KP1 * N; i += NT) s_acc[i] = src[i];
    } else {
        // acc = (0, X^{2N-barb} * [mu,...,mu])  (lwe-bootstrapping-functions-fft.cpp:142-145)
        const int e = 2 * N - my_bara[args.nsteps];
        for (int i = t; i < K * N; i += NT) s_acc[i] = 0u;
        for (int j = t; j < N; j += NT) {
            int src = j - e;
            uint32_t neg = 0;
            while (src < 0) {
                src += N;
                neg ^= 1u;
            }
            s_acc[K * N + j] = neg ? 0u - (uint32_t)args.mu : (uint32_t)args.mu;
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
    const T digit_bias = DigitConv<T>::base() + T(1 << (Bgbit - 1));

    int c = 0;  // key-row (chunk) counter, same sequence as the producer
    int a_next = (!EXT && args.nsteps > 0) ? my_bara[0] : 0;  // rotation amounts, loaded one step ahead
    // the new accumulator word: the old one plus the product, or (EXT) the product alone
    auto put = [](uint32_t &dst, uint32_t v) {
        if constexpr (EXT) dst = v;
        else dst += v;
    };
    for (int step = 0; step < args.nsteps; step++) {
        const int ai = a_next & (2 * N - 1);
        if (!EXT && step + 1 < args.nsteps) a_next = my_bara[step + 1];
        // FP64: one accumulator spectrum per output polynomial.  Split: hi- and lo-limb spectra as
        // packed register pairs over the slots (2m, 2m+1).
        cplx<T> acc_hi[SPLIT ? 1 : KP1][kR];
        cpair acc_h[SPLIT ? KP1 : 1][kR / 2], acc_l[SPLIT ? KP1 : 1][kR / 2];
        if constexpr (SPLIT) {
#pragma unroll
            for (int v = 0; v < KP1; v++)
#pragma unroll
                for (int m = 0; m < kR / 2; m++) {
                    acc_h[v][m] = {{0.f, 0.f}, {0.f, 0.f}};
                    acc_l[v][m] = {{0.f, 0.f}, {0.f, 0.f}};
                }
        } else {
#pragma unroll
            for (int v = 0; v < KP1; v++)
#pragma unroll
                for (int r = 0; r < kR; r++) acc_hi[v][r] = {T(0), T(0)};
        }

        // Two independent transforms side by side (two dependency chains for the scheduler) where
        // registers allow.  Inverse, at most 384 threads per CTA (168 registers each): the split form's
        // two limbs of one output (64.1 against 65.6 ms per 2048 bootstraps at N = 2048, G = 2), FP64's
        // two outputs.  At 128 registers the pair spills and ran 0.9 % slower (split, G = 7), so there
        // the transforms go one after the other.  Forward, FP64 at most 256 threads (255 registers):
        // the digits in chain order, two at a time, so every accumulator takes its products in the
        // same order as one at a time; the inverse that follows must be a pair (it begins with a
        // barrier).  One wave of 148 bootstraps at G = 1: 3.07 against 3.36 ms; at G = 3, 51.7 against
        // 53.6 ms per 4096.  The split form ran slower paired (3.97 against 3.20 ms at G = 1).
        constexpr bool kPairInverse = Lay::threads <= 384;
        constexpr bool kPairForward =
            !SPLIT && Lay::threads <= 256 && !Lay::rot_in_smem && KPL % 2 == 0 && kPairInverse && KP1 == 2;
        // one digit's spectrum times key row c into the accumulators; frees the row's ring slot
        auto accumulate = [&](const cplx<T> *z) {
            const int s = c % D;
            if constexpr (!PW) {
                // thread 0 issues every row before anyone waits for it
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
            const unsigned char *stage = smem + Lay::ring + (size_t)s * Lay::chunk;
            if constexpr (SPLIT) {
                // key row: [v][m][limb][t] x float4 {re(2m), re(2m+1), im(2m), im(2m+1)}
#pragma unroll
                for (int m = 0; m < kR / 2; m++) {
                    const cpair zp = make_cpair(z[2 * m], z[2 * m + 1]);
                    const float2 nzi = mul2(zp.im, make_float2(-1.f, -1.f));
#pragma unroll
                    for (int v = 0; v < KP1; v++) {
                        const float4 *kp = reinterpret_cast<const float4 *>(
                            stage + ((size_t)((v * (kR / 2) + m) * 2) * NT + t) * 16);
                        cmac_pair(acc_h[v][m], zp, nzi, kp[0]);
                        cmac_pair(acc_l[v][m], zp, nzi, kp[NT]);
                    }
                }
            } else {
#pragma unroll
                for (int v = 0; v < KP1; v++)
#pragma unroll
                    for (int r = 0; r < kR; r++) {
                        const size_t off = ((size_t)(v * kR + r) * NT + t) * 16;
                        const double2 b = *reinterpret_cast<const double2 *>(stage + off);
                        cmac(acc_hi[v][r], z[r], cplx<T>{(T)b.x, (T)b.y});
                    }
            }
            mbar_arrive(empty_bar(s));
            if constexpr (!PW) {
                while (issuing && issued < total_chunks && mbar_test_wait(empty_bar(issued % D), ((issued / D) - 1) & 1))
                    issue_row(issued++);
            }
            c++;
        };
        // digit q of the words x[r] (a_j) and x[kR + r] (a_{j+M}), j = t + NT * r
        auto decompose = [&](cplx<T> *z, const uint32_t *x, int q) {
            const int shift = 32 - (q + 1) * Bgbit;
#pragma unroll
            for (int r = 0; r < kR; r++) {
                const T d0 = DigitConv<T>::conv((x[r] >> shift) & maskBg, digit_bias);
                const T d1 = DigitConv<T>::conv((x[kR + r] >> shift) & maskBg, digit_bias);
                z[r] = cplx<T>{d0, -d1};  // a_j - i a_{j+M}; the twist is folded into the FFT
            }
        };

        if constexpr (kPairForward) {
            // every polynomial's (X^a - 1) * poly + offset in registers, then the digits two at a time
            uint32_t xr[KP1][2 * kR];
#pragma unroll
            for (int u = 0; u < KP1; u++)
#pragma unroll
                for (int r = 0; r < kR; r++) {
                    const int j = t + NT * r;
                    xr[u][r] = (EXT ? s_acc[u * N + j] : rot_minus_one<N>(s_acc + u * N, j, ai)) + offset;
                    xr[u][kR + r] = (EXT ? s_acc[u * N + j + M] : rot_minus_one<N>(s_acc + u * N, j + M, ai)) + offset;
                }
#pragma unroll 1
            for (int d = 0; d < KPL; d += 2) {
                cplx<T> za[kR], zb[kR];
                uint32_t x[2 * kR];
#pragma unroll
                for (int i = 0; i < 2 * kR; i++) {  // polynomial d / L (selects, no local memory)
                    x[i] = xr[0][i];
#pragma unroll
                    for (int u = 1; u < KP1; u++)
                        if (d / L == u) x[i] = xr[u][i];
                }
                decompose(za, x, d % L);
#pragma unroll
                for (int i = 0; i < 2 * kR; i++) {  // polynomial (d + 1) / L
                    x[i] = xr[0][i];
#pragma unroll
                    for (int u = 1; u < KP1; u++)
                        if ((d + 1) / L == u) x[i] = xr[u][i];
                }
                decompose(zb, x, (d + 1) % L);
                F::forward_pair(za, zb, xp, s_tw, t, bar_id);
                accumulate(za);
                accumulate(zb);
            }
        } else {
#pragma unroll 1
            for (int u = 0; u < KP1; u++) {
                const uint32_t *poly = s_acc + u * N;
                // (X^a - 1) * poly + offset, kept for the L digits: in the team's scratch (each thread
                // its own words, so no barrier, and no registers held across the digits' transforms)
                // or, where that does not fit, in registers
                uint32_t x[Lay::rot_in_smem ? 1 : 2 * kR];
#pragma unroll
                for (int r = 0; r < kR; r++) {
                    const int j = t + NT * r;
                    const uint32_t v0 = (EXT ? poly[j] : rot_minus_one<N>(poly, j, ai)) + offset;
                    const uint32_t v1 = (EXT ? poly[j + M] : rot_minus_one<N>(poly, j + M, ai)) + offset;
                    if constexpr (Lay::rot_in_smem) {
                        s_rot[r * NT + t] = v0;
                        s_rot[(kR + r) * NT + t] = v1;
                    } else {
                        x[r] = v0;
                        x[kR + r] = v1;
                    }
                }
#pragma unroll 1
                for (int q = 0; q < L; q++) {
                    const int shift = 32 - (q + 1) * Bgbit;
                    cplx<T> z[kR];
#pragma unroll
                    for (int r = 0; r < kR; r++) {
                        const uint32_t v0 = Lay::rot_in_smem ? s_rot[r * NT + t] : x[r];
                        const uint32_t v1 = Lay::rot_in_smem ? s_rot[(kR + r) * NT + t] : x[kR + r];
                        const T d0 = DigitConv<T>::conv((v0 >> shift) & maskBg, digit_bias);
                        const T d1 = DigitConv<T>::conv((v1 >> shift) & maskBg, digit_bias);
                        z[r] = cplx<T>{d0, -d1};  // a_j - i a_{j+M}; the twist is folded into the FFT
                    }
                    F::forward(z, xp, s_tw, t, bar_id);
                    accumulate(z);
                }
            }
        }

        // inverse transforms, exact rounding, accumulate (the key was pre-scaled by 1/M)
        if constexpr (!SPLIT && kPairInverse && KP1 == 2) {
            cplx<T> z0[kR], z1[kR];
#pragma unroll
            for (int r = 0; r < kR; r++) {
                z0[r] = acc_hi[0][r];
                z1[r] = acc_hi[1][r];
            }
            F::inverse_pair(z0, z1, xp, s_tw, t, bar_id);
#pragma unroll
            for (int r = 0; r < kR; r++) {
                const int j = t + NT * r;
                put(s_acc[j], round_f64_mod32(z0[r].re));  // (c_j - i c_{j+M})
                put(s_acc[j + M], round_f64_mod32(-z0[r].im));
                put(s_acc[N + j], round_f64_mod32(z1[r].re));
                put(s_acc[N + j + M], round_f64_mod32(-z1[r].im));
            }
        }
#pragma unroll
        for (int v = 0; v < KP1; v++) {
            if constexpr (!SPLIT && kPairInverse && KP1 == 2) break;  // done above
            uint32_t c0[kR], c1[kR];
            if constexpr (SPLIT && kPairInverse) {
                cplx<T> zh[kR], zl[kR];
#pragma unroll
                for (int m = 0; m < kR / 2; m++) {
                    zh[2 * m] = {acc_h[v][m].re.x, acc_h[v][m].im.x};
                    zh[2 * m + 1] = {acc_h[v][m].re.y, acc_h[v][m].im.y};
                    zl[2 * m] = {acc_l[v][m].re.x, acc_l[v][m].im.x};
                    zl[2 * m + 1] = {acc_l[v][m].re.y, acc_l[v][m].im.y};
                }
                F::inverse_pair(zh, zl, xp, s_tw, t, bar_id);
#pragma unroll
                for (int r = 0; r < kR; r++) {  // (c_j - i c_{j+M}) of each limb
                    c0[r] = (round_f32_mod32(zh[r].re) << args.split_shift) + (uint32_t)__float2ll_rn(zl[r].re);
                    c1[r] = (round_f32_mod32(-zh[r].im) << args.split_shift) + (uint32_t)__float2ll_rn(-zl[r].im);
                }
            } else if constexpr (SPLIT) {
                cplx<T> z[kR];
#pragma unroll
                for (int m = 0; m < kR / 2; m++) {
                    z[2 * m] = {acc_h[v][m].re.x, acc_h[v][m].im.x};
                    z[2 * m + 1] = {acc_h[v][m].re.y, acc_h[v][m].im.y};
                }
                F::inverse(z, xp, s_tw, t, bar_id);
#pragma unroll
                for (int r = 0; r < kR; r++) {
                    c0[r] = round_f32_mod32(z[r].re) << args.split_shift;
                    c1[r] = round_f32_mod32(-z[r].im) << args.split_shift;
                }
#pragma unroll
                for (int m = 0; m < kR / 2; m++) {
                    z[2 * m] = {acc_l[v][m].re.x, acc_l[v][m].im.x};
                    z[2 * m + 1] = {acc_l[v][m].re.y, acc_l[v][m].im.y};
                }
                F::inverse(z, xp, s_tw, t, bar_id);
#pragma unroll
                for (int r = 0; r < kR; r++) {
                    c0[r] += (uint32_t)__float2ll_rn(z[r].re);
                    c1[r] += (uint32_t)__float2ll_rn(-z[r].im);
                }
            } else {
                cplx<T> z[kR];
#pragma unroll
                for (int r = 0; r < kR; r++) z[r] = acc_hi[v][r];
                F::inverse(z, xp, s_tw, t, bar_id);
#pragma unroll
                for (int r = 0; r < kR; r++) {
                    c0[r] = round_f64_mod32(z[r].re);  // (c_j - i c_{j+M})
                    c1[r] = round_f64_mod32(-z[r].im);
                }
            }
            uint32_t *poly = s_acc + v * N;
#pragma unroll
            for (int r = 0; r < kR; r++) {
                const int j = t + NT * r;
                put(poly[j], c0[r]);
                put(poly[j + M], c1[r]);
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
}

// ---- one bootstrap per CTA, digits in parallel ------------------------------------------------
//
// Latency form for batches far below one wave (a single drop-in gate, a few concurrent callers): one
// CTA per bootstrap, one team per gadget digit ((k+1) * l teams of N/16 threads) plus the producer
// warp.  Per step:
//   1. team d rotates polynomial d / l, takes digit d % l and runs its forward transform; the spectra
//      go to shared memory;
//   2. jobs (output polynomial v, and in the split form the key limb) run on the first teams: the
//      multiply-accumulate over the digits in order 0..(k+1)l-1 against the key rows, then the inverse
//      transform, rounding and accumulation into the accumulator (split: the two limbs' teams add their
//      parts with shared-memory atomics; integer sums mod 2^32 are order-free).
// Each accumulator takes the same products in the same order as in blind_rotate_kernel, and each
// transform runs the same operations, so the results are bit-identical to it.
template <typename T, int N, int K, int L, int D, int XB>
struct WideLayout {
    static constexpr int M = N / 2, NT = M / kR, KP1 = K + 1, KPL = KP1 * L;
    static constexpr uint32_t chunk = (uint32_t)KP1 * M * 16;
    static constexpr size_t bars = 0;
    static constexpr size_t ring = (2 * D * 8 + 4 + 127) / 128 * 128;
    static constexpr size_t tables = ring + (size_t)D * chunk;
    static constexpr size_t tables_bytes = tw_table_bytes<T, M>();
    static constexpr size_t acc = (tables + tables_bytes + 127) / 128 * 128;
    static constexpr size_t spec = acc + 4 * (size_t)KP1 * N;           // [digit][slot] spectra
    static constexpr size_t spec_bytes = (size_t)KPL * M * 2 * sizeof(T);
    static constexpr size_t xbuf_bytes = ((size_t)Exch<T, M>::bytes + 15) / 16 * 16;
    static constexpr size_t xbufs = spec + spec_bytes;                   // [team][XB] exchange buffers
    static constexpr size_t bytes = xbufs + (size_t)KPL * XB * xbuf_bytes;
    static_assert(2 * D * 8 + 4 <= ring, "barrier block");
    static_assert(bytes <= 227 * 1024, "shared memory of the variant");
    static_assert(D >= 1 && (XB == 1 || XB == 2), "ring depth and exchange buffers");
};

template <typename T, int N, int K, int L, bool SPLIT, int D, int XB>
__global__ void __launch_bounds__((K + 1) * L * (N / 16) + 32, 1) blind_rotate_wide_kernel(const BrArgs args) {
    using Lay = WideLayout<T, N, K, L, D, XB>;
    constexpr int M = N / 2, NT = M / kR, KP1 = K + 1, KPL = KP1 * L;
    constexpr int JOBS = KP1 * (SPLIT ? 2 : 1);  // (output, limb) pairs
    static_assert(JOBS <= KPL, "every job needs a team");
    using F = TeamFft<T, M, kR>;
    extern __shared__ __align__(128) unsigned char smem[];

    const int tid = threadIdx.x;
    constexpr int consumers = KPL * NT;
    constexpr int kAllBar = 15;  // named barrier of all consumer teams (teams use 1..KPL)
    static_assert(KPL < kAllBar, "named barrier ids");
    const uint32_t bar0 = smem_addr(smem + Lay::bars);
    auto full_bar = [&](int s) { return bar0 + 8u * s; };
    auto empty_bar = [&](int s) { return bar0 + 8u * (D + s); };
    volatile int32_t *abort_flag = reinterpret_cast<volatile int32_t *>(smem + Lay::bars + 16 * D);
    const uint32_t ring = smem_addr(smem + Lay::ring);

    if (tid == 0) {
        for (int s = 0; s < D; s++) {
            mbar_init(full_bar(s), 1);
            mbar_init(empty_bar(s), (uint32_t)(JOBS * NT));
        }
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    {
        const int4 *g_tab = reinterpret_cast<const int4 *>(args.tables);
        int4 *s_tab4 = reinterpret_cast<int4 *>(smem + Lay::tables);
        for (int i = tid; i < (int)(Lay::tables_bytes / 16); i += blockDim.x) s_tab4[i] = g_tab[i];
    }
    __syncthreads();

    const int total_chunks = args.nsteps * KPL;
    if (tid >= consumers) {  // producer warp: stream the key rows, as in blind_rotate_kernel
        if (tid == consumers) {
            int issued = 0;
            if (!args.stall_producer) {
                for (int c = 0; c < total_chunks; c++) {
                    const int s = c % D;
                    if (c >= D && !wait_bounded(empty_bar(s), ((c / D) - 1) & 1, abort_flag, args.timeout_ns, args.err))
                        break;
                    mbar_arrive_expect_tx(full_bar(s), Lay::chunk);
                    bulk_copy_g2s(ring + (uint32_t)s * Lay::chunk, args.bsk + (size_t)c * Lay::chunk, Lay::chunk,
                                  full_bar(s));
                    issued = c + 1;
                }
            }
            volatile int32_t no_abort = 0;
            for (int c = (issued > D ? issued - D : 0); c < issued; c++)
                wait_bounded(full_bar(c % D), (c / D) & 1, &no_abort, args.timeout_ns, args.err);
        }
        return;
    }

    const int team = tid / NT;  // digit of the forward phase; job of the accumulate phase
    const int t = tid - team * NT;
    const int bar_id = 1 + team;
    const int boot = blockIdx.x;
    uint32_t *s_acc = reinterpret_cast<uint32_t *>(smem + Lay::acc);
    T *s_spec = reinterpret_cast<T *>(smem + Lay::spec);
    ExchPair xp{smem + Lay::xbufs + (size_t)team * XB * Lay::xbuf_bytes, XB == 2 ? (uint32_t)Lay::xbuf_bytes : 0u,
                0u};
    const cplx<T> *s_tw = reinterpret_cast<const cplx<T> *>(smem + Lay::tables);

    const int32_t *my_bara = args.bara + (size_t)boot * args.bara_stride;
    if (args.acc_in) {
        const uint32_t *src = reinterpret_cast<const uint32_t *>(args.acc_in) + (size_t)boot * KP1 * N;
        for (int i = tid; i < KP1 * N; i += consumers) s_acc[i] = src[i];
    } else {
        // acc = (0, X^{2N-barb} * [mu,...,mu])  (lwe-bootstrapping-functions-fft.cpp:142-145)
        const int e = 2 * N - my_bara[args.nsteps];
        for (int i = tid; i < K * N; i += consumers) s_acc[i] = 0u;
        for (int j = tid; j < N; j += consumers) {
            int src = j - e;
            uint32_t neg = 0;
            while (src < 0) {
                src += N;
                neg ^= 1u;
            }
            s_acc[K * N + j] = neg ? 0u - (uint32_t)args.mu : (uint32_t)args.mu;
        }
    }
    team_sync(kAllBar, consumers);

    // gadget constants (tgsw.cpp:7-29)
    const int Bgbit = args.Bgbit;
    uint32_t offset = 0;
#pragma unroll
    for (int q = 0; q < L; q++) offset += 1u << (32 - (q + 1) * Bgbit);
    offset *= 1u << (Bgbit - 1);
    const uint32_t maskBg = (1u << Bgbit) - 1u;
    const T digit_bias = DigitConv<T>::base() + T(1 << (Bgbit - 1));
    const int u_poly = team / L;                     // polynomial of this team's digit
    const int shift = 32 - (team - u_poly * L + 1) * Bgbit;

    int c = 0;  // first key row of the step
    int a_next = args.nsteps > 0 ? my_bara[0] : 0;
    for (int step = 0; step < args.nsteps; step++, c += KPL) {
        const int ai = a_next & (2 * N - 1);
        if (step + 1 < args.nsteps) a_next = my_bara[step + 1];

        // 1. this team's digit: (X^a - 1) * poly + offset, digit, forward transform, spectrum out
        {
            const uint32_t *poly = s_acc + u_poly * N;
            cplx<T> z[kR];
#pragma unroll
            for (int r = 0; r < kR; r++) {
                const int j = t + NT * r;
                const uint32_t v0 = rot_minus_one<N>(poly, j, ai) + offset;
                const uint32_t v1 = rot_minus_one<N>(poly, j + M, ai) + offset;
                const T d0 = DigitConv<T>::conv((v0 >> shift) & maskBg, digit_bias);
                const T d1 = DigitConv<T>::conv((v1 >> shift) & maskBg, digit_bias);
                z[r] = cplx<T>{d0, -d1};  // a_j - i a_{j+M}; the twist is folded into the FFT
            }
            F::forward(z, xp, s_tw, t, bar_id);
            if constexpr (SPLIT) {
                // [digit][m][t] float4 {re(2m), re(2m+1), im(2m), im(2m+1)}
                float4 *sp = reinterpret_cast<float4 *>(s_spec) + (size_t)team * (kR / 2) * NT + t;
#pragma unroll
                for (int m = 0; m < kR / 2; m++)
                    sp[m * NT] = make_float4(z[2 * m].re, z[2 * m + 1].re, z[2 * m].im, z[2 * m + 1].im);
            } else {
                double2 *sp = reinterpret_cast<double2 *>(s_spec) + (size_t)team * kR * NT + t;
#pragma unroll
                for (int r = 0; r < kR; r++) sp[r * NT] = make_double2(z[r].re, z[r].im);
            }
        }
        team_sync(kAllBar, consumers);

        // 2. job `team`: multiply-accumulate over the digits in order, inverse transform, accumulate
        if (team < JOBS) {
            const int v = SPLIT ? team >> 1 : team;
            if constexpr (SPLIT) {
                const int limb = team & 1;
                cpair acc[kR / 2];
#pragma unroll
                for (int m = 0; m < kR / 2; m++) acc[m] = {{0.f, 0.f}, {0.f, 0.f}};
#pragma unroll
                for (int d = 0; d < KPL; d++) {
                    const int row = c + d, s = row % D;
                    wait_bounded(full_bar(s), (row / D) & 1, abort_flag, args.timeout_ns, args.err);
                    const float4 *kp = reinterpret_cast<const float4 *>(smem + Lay::ring + (size_t)s * Lay::chunk);
                    const float4 *sp = reinterpret_cast<const float4 *>(s_spec) + (size_t)d * (kR / 2) * NT + t;
#pragma unroll
                    for (int m = 0; m < kR / 2; m++) {
                        const float4 f = sp[m * NT];
                        const cpair zp{{f.x, f.y}, {f.z, f.w}};
                        const float2 nzi = mul2(zp.im, make_float2(-1.f, -1.f));
                        cmac_pair(acc[m], zp, nzi, kp[((v * (kR / 2) + m) * 2 + limb) * NT + t]);
                    }
                    mbar_arrive(empty_bar(s));
                }
                cplx<T> z[kR];
#pragma unroll
                for (int m = 0; m < kR / 2; m++) {
                    z[2 * m] = {acc[m].re.x, acc[m].im.x};
                    z[2 * m + 1] = {acc[m].re.y, acc[m].im.y};
                }
                F::inverse(z, xp, s_tw, t, bar_id);
                uint32_t *poly = s_acc + v * N;
#pragma unroll
                for (int r = 0; r < kR; r++) {  // (c_j - i c_{j+M}) of this limb
                    const int j = t + NT * r;
                    const uint32_t c0 = limb == 0 ? round_f32_mod32(z[r].re) << args.split_shift
                                                  : (uint32_t)__float2ll_rn(z[r].re);
                    const uint32_t c1 = limb == 0 ? round_f32_mod32(-z[r].im) << args.split_shift
                                                  : (uint32_t)__float2ll_rn(-z[r].im);
                    atomicAdd(poly + j, c0);
                    atomicAdd(poly + j + M, c1);
                }
            } else {
                cplx<T> acc[kR];
#pragma unroll
                for (int r = 0; r < kR; r++) acc[r] = {T(0), T(0)};
#pragma unroll
                for (int d = 0; d < KPL; d++) {
                    const int row = c + d, s = row % D;
                    wait_bounded(full_bar(s), (row / D) & 1, abort_flag, args.timeout_ns, args.err);
                    const double2 *kp = reinterpret_cast<const double2 *>(smem + Lay::ring + (size_t)s * Lay::chunk);
                    const double2 *sp = reinterpret_cast<const double2 *>(s_spec) + (size_t)d * kR * NT + t;
#pragma unroll
                    for (int r = 0; r < kR; r++) {
                        const double2 zz = sp[r * NT];
                        const double2 b = kp[(v * kR + r) * NT + t];
                        cmac(acc[r], cplx<T>{(T)zz.x, (T)zz.y}, cplx<T>{(T)b.x, (T)b.y});
                    }
                    mbar_arrive(empty_bar(s));
                }
                F::inverse(acc, xp, s_tw, t, bar_id);
                uint32_t *poly = s_acc + v * N;
#pragma unroll
                for (int r = 0; r < kR; r++) {
                    const int j = t + NT * r;
                    poly[j] += round_f64_mod32(acc[r].re);  // (c_j - i c_{j+M})
                    poly[j + M] += round_f64_mod32(-acc[r].im);
                }
            }
        }
        team_sync(kAllBar, consumers);
    }

    uint32_t *dst = reinterpret_cast<uint32_t *>(args.acc_out) + (size_t)boot * KP1 * N;
    for (int i = tid; i < KP1 * N; i += consumers) dst[i] = s_acc[i];
}

// ---- launch -------------------------------------------------------------------------------------

template <typename T, int N, int L, bool SPLIT, int G, int D, bool PW = true>
static cudaError_t launch_g(const BrArgs &a, cudaStream_t s) {
    using Lay = BrLayout<T, N, 1, G, D, PW>;
    const size_t smem = Lay::bytes(a.nsteps);
    auto kern = blind_rotate_kernel<T, N, 1, L, SPLIT, G, D, PW>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int grid = (a.boots + G - 1) / G;
    kern<<<grid, Lay::threads, smem, s>>>(a);
    return cudaGetLastError();
}

template <typename T, int N, int L, bool SPLIT, int D, int XB>
static cudaError_t launch_wide(const BrArgs &a, cudaStream_t s) {
    using Lay = WideLayout<T, N, 1, L, D, XB>;
    auto kern = blind_rotate_wide_kernel<T, N, 1, L, SPLIT, D, XB>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)Lay::bytes);
    if (e != cudaSuccess) return e;
    kern<<<a.boots, 2 * L * (N / 16) + 32, Lay::bytes, s>>>(a);
    return cudaGetLastError();
}

// External product only (EXT), one sample per CTA, thread 0 streaming the key rows.
template <typename T, int N, int L, bool SPLIT, int D>
static cudaError_t launch_ext(const BrArgs &a, cudaStream_t s) {
    using Lay = BrLayout<T, N, 1, 1, D, false>;
    const size_t smem = Lay::bytes(a.nsteps);
    auto kern = blind_rotate_kernel<T, N, 1, L, SPLIT, 1, D, false, true>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    kern<<<a.boots, Lay::threads, smem, s>>>(a);
    return cudaGetLastError();
}

int blind_rotate_supported(const tfheb_params &p) {
    return br_variants(p.N, p.l, p.k == 1 ? TFHEB_FP64 : -1, nullptr, nullptr, 0) > 0;
}

// Compiled launch variants: (ring degree, precision, bootstraps per CTA G, key-ring depth D, and
// whether a producer warp streams the key; without it, thread 0 does).
// Every variant's shared memory stays within 227 KB.  Tuned variants are the autotuner's candidates:
// the first of a (N, l, precision) triple is the default, and tfheb_autotune times all of them on the
// device and keeps the fastest per key.  Small variants (few bootstraps per CTA) serve batches that
// fit one wave of CTAs with fewer bootstraps per SM than the tuned variant would pack (see
// launch_blind_rotate).
struct BrVariant {
    int N, l, precision, G, D;
    bool tuned;
    cudaError_t (*launch)(const BrArgs &, cudaStream_t);
    int plan = 0;  // 0: one transform per thread; 1: two per thread, spectra in TMEM (blind_rotate_paired.cu)
};
static const BrVariant kBrVariants[] = {
    // the split default: two transforms per thread, spectra in TMEM, a 12-half-row key ring; the
    // step's rotated words wait in TMEM, the first two digit pairs' forward transforms run
    // interleaved, and so do both outputs' inverse transforms, output 0's input waiting in TMEM
    // meanwhile; the keys of a digit's first two slot pairs load during the previous digit's
    // multiply-accumulate (30.94 ms per 4096 bootstraps, no spills; on another box 31.50 against
    // 31.33 ms without it, so both stay candidates and the autotuner picks).  The same kernel
    // without that prefetch: 31.27 ms; loading 3 or 4 slot pairs ahead: 31.49 / 31.68 ms; with less interleaving: 31.59 ms (inverse input in registers, 20 B of
    // spills), 31.85 ms (forward only), 32.2 ms (none, rotated words in registers); 36.24 ms for the
    // plan-0 G = 7, D = 6 below.
    {1024, 3, TFHEB_SPLIT_FP32, 7, 12, true, launch_paired_il7<1024, 3, 7, 12, 1>, 1},
    {1024, 3, TFHEB_SPLIT_FP32, 7, 12, true, launch_paired_il3<1024, 3, 7, 12, 1>, 1},
    {1024, 3, TFHEB_SPLIT_FP32, 7, 12, true, launch_paired_il2<1024, 3, 7, 12, 1>, 1},
    {1024, 3, TFHEB_SPLIT_FP32, 7, 12, true, launch_paired_il<1024, 3, 7, 12, 1>, 1},
    {1024, 3, TFHEB_SPLIT_FP32, 7, 12, true, launch_paired<1024, 3, 7, 12, 1, true>, 1},
    {1024, 3, TFHEB_SPLIT_FP32, 7, 6, true, launch_g<float, 1024, 3, true, 7, 6>},
    {1024, 3, TFHEB_SPLIT_FP32, 7, 4, true, launch_g<float, 1024, 3, true, 7, 4>},
    {1024, 3, TFHEB_SPLIT_FP32, 5, 4, true, launch_g<float, 1024, 3, true, 5, 4>},
    {1024, 3, TFHEB_SPLIT_FP32, 4, 4, true, launch_g<float, 1024, 3, true, 4, 4>},
    // plan 1: D counts half rows (8 KB) here; single or double exchange buffers per team
    {1024, 3, TFHEB_SPLIT_FP32, 7, 8, true, launch_paired<1024, 3, 7, 8, 1, true>, 1},
    {1024, 3, TFHEB_SPLIT_FP32, 7, 4, true, launch_paired<1024, 3, 7, 4, 2, true>, 1},
    {1024, 3, TFHEB_SPLIT_FP32, 6, 6, true, launch_paired<1024, 3, 6, 6, 2, true>, 1},
    {1024, 3, TFHEB_SPLIT_FP32, 3, 4, false, launch_g<float, 1024, 3, true, 3, 4>},
    {1024, 3, TFHEB_SPLIT_FP32, 2, 4, false, launch_g<float, 1024, 3, true, 2, 4>},
    {1024, 3, TFHEB_SPLIT_FP32, 1, 4, false, launch_g<float, 1024, 3, true, 1, 4>},
    // the default's kernel with 3-6 teams, for batches of one wave (later than plan 0's equals, so
    // the default small-batch rule takes them): one wave of 148 G bootstraps in 4.78 / 5.03 / 6.12 /
    // 6.59 ms at G = 3 / 4 / 5 / 6, against 5.64 (G = 4) and 6.85 ms (G = 5) for plan 0
    {1024, 3, TFHEB_SPLIT_FP32, 6, 12, false, launch_paired_il3<1024, 3, 6, 12, 1>, 1},
    {1024, 3, TFHEB_SPLIT_FP32, 5, 12, false, launch_paired_il3<1024, 3, 5, 12, 1>, 1},
    {1024, 3, TFHEB_SPLIT_FP32, 4, 12, false, launch_paired_il3<1024, 3, 4, 12, 1>, 1},
    {1024, 3, TFHEB_SPLIT_FP32, 3, 12, false, launch_paired_il3<1024, 3, 3, 12, 1>, 1},
    {1024, 3, TFHEB_SPLIT_FP32, 1, 8, false, launch_wide<float, 1024, 3, true, 8, 2>},
    {1024, 3, TFHEB_FP64, 4, 5, true, launch_g<double, 1024, 3, false, 4, 5, false>},
    {1024, 3, TFHEB_FP64, 4, 4, true, launch_g<double, 1024, 3, false, 4, 4, false>},
    {1024, 3, TFHEB_FP64, 4, 6, true, launch_g<double, 1024, 3, false, 4, 6>},
    {1024, 3, TFHEB_FP64, 4, 4, true, launch_g<double, 1024, 3, false, 4, 4>},
    {1024, 3, TFHEB_FP64, 3, 4, true, launch_g<double, 1024, 3, false, 3, 4>},
    {1024, 3, TFHEB_FP64, 2, 4, true, launch_g<double, 1024, 3, false, 2, 4>},
    {1024, 3, TFHEB_FP64, 1, 4, false, launch_g<double, 1024, 3, false, 1, 4>},
    {1024, 3, TFHEB_FP64, 1, 6, false, launch_wide<double, 1024, 3, false, 6, 1>},
    // the split default at N = 2048: the N = 1024 default's structure with three teams and a 6-deep
    // ring of 16 KB half rows (51.3 ms per 2048 bootstraps; 51.7 ms with output 0's inverse input in
    // registers, 51.9 ms forward interleave only, 53.1 ms no interleave, 54.1 ms rotated words in
    // registers too, 56.5 ms 4 deep, 62.6 ms for the plan-0 G = 2 below)
    {2048, 3, TFHEB_SPLIT_FP32, 3, 6, true, launch_paired_il3<2048, 3, 3, 6, 1>, 1},
    {2048, 3, TFHEB_SPLIT_FP32, 3, 6, true, launch_paired_il2<2048, 3, 3, 6, 1>, 1},
    {2048, 3, TFHEB_SPLIT_FP32, 3, 6, true, launch_paired_il<2048, 3, 3, 6, 1>, 1},
    {2048, 3, TFHEB_SPLIT_FP32, 3, 4, true, launch_paired<2048, 3, 3, 4, 1, true>, 1},
    {2048, 3, TFHEB_SPLIT_FP32, 2, 4, true, launch_g<float, 2048, 3, true, 2, 4, false>},
    {2048, 3, TFHEB_SPLIT_FP32, 2, 4, true, launch_g<float, 2048, 3, true, 2, 4>},
    {2048, 3, TFHEB_SPLIT_FP32, 3, 3, true, launch_g<float, 2048, 3, true, 3, 3>},
    {2048, 3, TFHEB_SPLIT_FP32, 2, 3, true, launch_g<float, 2048, 3, true, 2, 3>},
    {2048, 3, TFHEB_SPLIT_FP32, 1, 3, false, launch_g<float, 2048, 3, true, 1, 3>},
    {2048, 3, TFHEB_SPLIT_FP32, 2, 4, true, launch_paired<2048, 3, 2, 4, 2, false>, 1},
    {2048, 3, TFHEB_SPLIT_FP32, 2, 4, true, launch_paired<2048, 3, 2, 4, 2, true>, 1},
    {2048, 3, TFHEB_FP64, 2, 3, true, launch_g<double, 2048, 3, false, 2, 3, false>},
    {2048, 3, TFHEB_FP64, 2, 3, true, launch_g<double, 2048, 3, false, 2, 3>},
    {2048, 3, TFHEB_FP64, 1, 4, true, launch_g<double, 2048, 3, false, 1, 4>},
    {512, 3, TFHEB_SPLIT_FP32, 8, 4, true, launch_g<float, 512, 3, true, 8, 4>},
    {512, 3, TFHEB_FP64, 8, 4, true, launch_g<double, 512, 3, false, 8, 4>},
    // the 80-bit parameter set (n = 500, l = 2, Bgbit = 10; tfhe_gate_bootstrapping.cpp:23-48)
    {1024, 2, TFHEB_SPLIT_FP32, 7, 4, true, launch_g<float, 1024, 2, true, 7, 4>},
    {1024, 2, TFHEB_SPLIT_FP32, 1, 4, false, launch_g<float, 1024, 2, true, 1, 4>},
    {1024, 2, TFHEB_SPLIT_FP32, 1, 8, false, launch_wide<float, 1024, 2, true, 8, 2>},
    {1024, 2, TFHEB_FP64, 4, 4, true, launch_g<double, 1024, 2, false, 4, 4, false>},
    {1024, 2, TFHEB_FP64, 4, 4, true, launch_g<double, 1024, 2, false, 4, 4>},
    {1024, 2, TFHEB_FP64, 1, 4, false, launch_g<double, 1024, 2, false, 1, 4>},
    {1024, 2, TFHEB_FP64, 1, 6, false, launch_wide<double, 1024, 2, false, 6, 2>},
};

int br_variants(int N, int l, int precision, int *G, int *D, int cap) {
    int n = 0;
    for (const auto &v : kBrVariants)
        if (v.tuned && v.N == N && v.l == l && v.precision == precision) {
            if (n < cap) {
                if (G) G[n] = v.G;
                if (D) D[n] = v.D;
            }
            n++;
        }
    return n;
}

static BrArgs br_args(const tfheb_params &p, const DeviceBsk &bsk, const int32_t *bara, int bara_stride, int boots,
                      int nsteps, int32_t mu, const int32_t *acc_in, int32_t *acc_out, int32_t *d_err,
                      int stall_producer, uint64_t timeout_ns) {
    return BrArgs{bara,       bara_stride, reinterpret_cast<const uint8_t *>(bsk.bsk), bsk.tables, bsk.tables2, acc_in,
                  acc_out,    boots,       nsteps, mu, p.Bgbit, bsk.split_shift, d_err, timeout_ns, stall_producer};
}

int br_variant_count() { return (int)(sizeof(kBrVariants) / sizeof(kBrVariants[0])); }

void br_variant_info(int g, int *N, int *l, int *precision, int *G, int *D, int *tuned) {
    const BrVariant &v = kBrVariants[g];
    if (N) *N = v.N;
    if (l) *l = v.l;
    if (precision) *precision = v.precision;
    if (G) *G = v.G;
    if (D) *D = v.D;
    if (tuned) *tuned = v.tuned;
}

int br_variant_plan(int g) { return kBrVariants[g].plan; }

int br_variant_plans(int N, int l, int precision, int *plan, int cap) {
    int n = 0;
    for (const auto &v : kBrVariants)
        if (v.tuned && v.N == N && v.l == l && v.precision == precision) {
            if (plan && n < cap) plan[n] = v.plan;
            n++;
        }
    return n;
}

int br_tuned_global(int N, int l, int precision, int tuned) {
    int seen = 0;
    for (int g = 0; g < br_variant_count(); g++) {
        const BrVariant &v = kBrVariants[g];
        if (v.tuned && v.N == N && v.l == l && v.precision == precision && seen++ == tuned) return g;
    }
    return -1;
}

cudaError_t launch_blind_rotate_exact(const tfheb_params &p, int precision, const DeviceBsk &bsk, const int32_t *bara,
                                      int bara_stride, int boots, int nsteps, int32_t mu, const int32_t *acc_in,
                                      int32_t *acc_out, cudaStream_t s, int32_t *d_err, int stall_producer,
                                      uint64_t timeout_ns, int global_index) {
    if (boots <= 0) return cudaSuccess;
    if (global_index < 0 || global_index >= br_variant_count()) return cudaErrorInvalidValue;
    const BrVariant &v = kBrVariants[global_index];
    if (v.N != p.N || v.l != p.l || v.precision != precision) return cudaErrorInvalidValue;
    return v.launch(br_args(p, bsk, bara, bara_stride, boots, nsteps, mu, acc_in, acc_out, d_err, stall_producer,
                            timeout_ns), s);
}

cudaError_t launch_blind_rotate(const tfheb_params &p, int precision, const DeviceBsk &bsk, const int32_t *bara,
                                int bara_stride, int boots, int nsteps, int32_t mu, const int32_t *acc_in,
                                int32_t *acc_out, cudaStream_t s, int32_t *d_err, int stall_producer,
                                uint64_t timeout_ns, const BrChoice &choice) {
    if (boots <= 0) return cudaSuccess;
    int g = br_tuned_global(p.N, p.l, precision, choice.tuned);
    if (g < 0) return cudaErrorInvalidValue;
    // A batch that fits one wave of CTAs with fewer bootstraps per CTA than the tuned variant packs
    // may run faster spread thinner: at the default parameters a lone split-FP32 team finishes its
    // 630 steps in 2.9 ms, while seven sharing an SM take 9.3 ms, so 16 gates packed 7 per CTA onto 3
    // SMs would wait for the busiest of them.  FP64: 148 gates in 3.1 ms one per CTA, 7.3 ms four per
    // CTA.
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) == cudaSuccess &&
        sms > 0) {
        const int need = (boots + sms - 1) / sms;  // bootstraps per CTA for one wave
        if (need < kBrVariants[g].G && need < kSmallNeeds) {
            const int e = choice.small[need];
            if (e >= 0 && e < br_variant_count()) {
                g = e;
            } else if (e == -2) {  // fewest bootstraps per CTA that fit; of equals, the later entry
                int pick = -1;
                for (int i = 0; i < br_variant_count(); i++) {
                    const BrVariant &v = kBrVariants[i];
                    if (v.N == p.N && v.l == p.l && v.precision == precision && v.G >= need &&
                        v.G < kBrVariants[g].G && (pick < 0 || v.G <= kBrVariants[pick].G))
                        pick = i;
                }
                if (pick >= 0) g = pick;
            }
        }
    }
    return launch_blind_rotate_exact(p, precision, bsk, bara, bara_stride, boots, nsteps, mu, acc_in, acc_out, s, d_err,
                                     stall_producer, timeout_ns, g);
}

struct ExtVariant {
    int N, l, precision;
    cudaError_t (*launch)(const BrArgs &, cudaStream_t);
};
static const ExtVariant kExtVariants[] = {
    {1024, 3, TFHEB_FP64, launch_ext<double, 1024, 3, false, 3>},
    {1024, 3, TFHEB_SPLIT_FP32, launch_ext<float, 1024, 3, true, 3>},
    {1024, 2, TFHEB_FP64, launch_ext<double, 1024, 2, false, 3>},
    {1024, 2, TFHEB_SPLIT_FP32, launch_ext<float, 1024, 2, true, 3>},
    {2048, 3, TFHEB_FP64, launch_ext<double, 2048, 3, false, 3>},
    {2048, 3, TFHEB_SPLIT_FP32, launch_ext<float, 2048, 3, true, 3>},
    {512, 3, TFHEB_FP64, launch_ext<double, 512, 3, false, 3>},
    {512, 3, TFHEB_SPLIT_FP32, launch_ext<float, 512, 3, true, 3>},
};

cudaError_t launch_extern_product(const tfheb_params &p, int precision, const DeviceBsk &bsk, int count,
                                  const int32_t *in, int32_t *out, cudaStream_t s, int32_t *d_err,
                                  uint64_t timeout_ns) {
    if (count <= 0) return cudaSuccess;
    if (!in || !out) return cudaErrorInvalidValue;
    for (const auto &v : kExtVariants)
        if (v.N == p.N && v.l == p.l && v.precision == precision)
            return v.launch(br_args(p, bsk, nullptr, 0, count, 1, 0, in, out, d_err, 0, timeout_ns), s);
    return cudaErrorInvalidValue;
}

}  // namespace tfheb
