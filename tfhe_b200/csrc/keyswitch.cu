// keyswitch.cu -- integer keyswitch on sm_100a (lweKeySwitchTranslate_fromArray,
// lwe-keyswitch-functions.cpp:114-141, and lweKeySwitch :225-238).
//
// For every extracted sample (a, b) of dimension kN the keyswitch forms
//     out = (0, b) - sum_{i < kN, j < t} ks[i][j][digit_j(a_i + 2^(31 - t*basebit))]
// with digit_j the j-th basebit-bit digit from the top.  All arithmetic is mod 2^32, so any order of
// the additions gives the reference's result bit for bit.
//
// Three CUDA-core kernels here, and the tensor-core kernel of keyswitch_mma.cu (the default wherever
// t = 8 and basebit = 2; the three below remain as cross-checks and for other digit shapes):
//   keyswitch_gate_kernel   one CTA per sample, each thread 4 output columns; the selected key rows are
//                           gathered from L2 per sample (15.5 MB of rows per sample at n = 630).  Used
//                           for parameter sets without a tiled instantiation, or on request.
//   keyswitch_tiled_kernel  one CTA per (64 samples, slice of 4*CW output columns, range of i).  The key
//                           rows of one input coefficient i (t x 3 non-zero digits x slice) are copied
//                           into a shared-memory ring by the TMA engine (cp.async.bulk, no multicast)
//                           and reused by all 64 samples; lane = sample, so the 32 lanes of a warp read
//                           at most 4 distinct rows (digit 0 reads a zero row) and every 16-byte load
//                           is a broadcast.  L2->SM key traffic drops from 15.5 MB per sample to 15.5 MB
//                           per 64 samples.  Small batches split the i range over CTAs and combine the
//                           partial sums with atomic adds (mod 2^32, exact).
//   keyswitch_regkey_kernel lane = column pair, key rows of one (i, j) held in registers and applied to
//                           7 samples per warp through a warp-uniform digit branch; each loaded key
//                           word serves 7 subtractions.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

#include "async_copy.cuh"
#include "internal.h"

namespace tfheb {

// ============================================================================================
// per-sample kernel
// ============================================================================================

// One CTA per sample; thread owns 4 consecutive output coefficients (int4 loads of the key rows).
// ksk rows: [kN][t][base][ks_stride], ks_stride a multiple of 4, zero padded.
__global__ void __launch_bounds__(256) keyswitch_gate_kernel(const int32_t *__restrict__ ksk, int ks_stride,
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

// ============================================================================================
// tiled kernel
// ============================================================================================

constexpr int kKsT = 8;                    // digits per coefficient (ks_t)
constexpr int kKsBase = 4;                 // 2^basebit
constexpr int kKsGateWarps = 2;            // warps along the samples of a tile
constexpr int kKsColWarps = 4;             // warps along the columns of a slice
constexpr int kKsThreads = 32 * kKsGateWarps * kKsColWarps;
constexpr int kKsTile = 32 * kKsGateWarps;  // samples per CTA
constexpr int kKsChunk = 32;               // input coefficients staged per refill of the mask tile
constexpr int kKsCws[] = {40, 52};         // compiled columns-per-warp choices

template <int CW>
struct KsTiled {
    static_assert(CW % 4 == 0, "columns per warp must be a multiple of 4 (16-byte loads)");
    static constexpr int slice = kKsColWarps * CW;  // output columns per CTA
    // Row stride in words.  4*(CW+1) with CW+1 odd puts the four digit rows of one column into four
    // disjoint 4-bank windows, so a warp's broadcast 16-byte loads never conflict.
    static constexpr int rs = slice + 4;
    static constexpr int stage_words = kKsT * kKsBase * rs;  // [j][digit 0..3][rs]; digit 0 row stays 0
    static constexpr int stage_bytes = 4 * stage_words;
    static constexpr int copy_bytes = 4 * (kKsBase - 1) * rs;  // digits 1..3 of one j (contiguous)
    static constexpr int block_words = kKsT * (kKsBase - 1) * rs;  // global words per (slice, i)
    static constexpr int stages = 3;
    static constexpr int sa_ld = kKsTile + 1;
    static constexpr int ring_off = 128;  // [0, 24): full barriers, [64]: abort flag
    static constexpr int sa_off = ring_off + stages * stage_bytes;
    static constexpr int smem_bytes = sa_off + 4 * kKsChunk * sa_ld;
    static_assert(copy_bytes % 16 == 0 && stage_bytes % 16 == 0, "bulk copies need 16-byte sizes");
    static_assert((kKsBase * rs * 4) % 16 == 0 && (rs * 4) % 16 == 0, "bulk copy destinations 16-byte aligned");
    static_assert(kKsGateWarps * kKsColWarps * 32 * (CW + 1) * 4 <= stages * stage_bytes,
                  "output transpose must fit in the ring");
};

template <int CW>
__global__ void __launch_bounds__(kKsThreads, 2)
    keyswitch_tiled_kernel(const int32_t *__restrict__ tiles, const uint32_t *__restrict__ in, int in_stride,
                           uint32_t *__restrict__ out, int count, int n, int kN, int slices, int ksplit,
                           int chunk_len, uint64_t timeout_ns, int32_t *err, int stall) {
    using L = KsTiled<CW>;
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int gw = warp / kKsColWarps, cw = warp - gw * kKsColWarps;
    const int kchunk = blockIdx.x % ksplit;
    const int unit = blockIdx.x / ksplit;
    const int slice = unit % slices, tile = unit / slices;
    const int i_begin = kchunk * chunk_len;
    const int i_count = min(kN, i_begin + chunk_len) - i_begin;

    const uint32_t bars = smem_addr(smem);
    volatile int32_t *abort_flag = reinterpret_cast<volatile int32_t *>(smem + 64);
    uint32_t *ring = reinterpret_cast<uint32_t *>(smem + L::ring_off);
    uint32_t *s_a = reinterpret_cast<uint32_t *>(smem + L::sa_off);

    if (tid == 0) {
        for (int s = 0; s < L::stages; s++) mbar_init(bars + 8 * s, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // the digit-0 rows are never written by the copies: zero them once
    for (int e = tid; e < L::stages * kKsT * L::rs; e += kKsThreads) {
        const int row = e / L::rs, c = e - row * L::rs;
        ring[row * kKsBase * L::rs + c] = 0;
    }
    __syncthreads();

    const int32_t *src = tiles + ((size_t)slice * kN + i_begin) * L::block_words;
    auto issue = [&](int q, int s) {
        const uint32_t bar = bars + 8 * s;
        mbar_arrive_expect_tx(bar, kKsT * L::copy_bytes);
        const int32_t *blk = src + (size_t)q * L::block_words;
        const uint32_t dst = smem_addr(ring + s * L::stage_words + L::rs);
#pragma unroll
        for (int j = 0; j < kKsT; j++)
            bulk_copy_g2s(dst + j * kKsBase * L::rs * 4, blk + j * (kKsBase - 1) * L::rs, L::copy_bytes, bar);
    };
    int issued = 0;  // meaningful in thread 0 only
    if (tid == 0 && !stall)  // stall: failure-detection test hook, no copy is ever issued
        for (; issued < L::stages && issued < i_count; issued++) issue(issued, issued);

    uint32_t acc[CW];
#pragma unroll
    for (int c = 0; c < CW; c++) acc[c] = 0;
    const int gl = gw * 32 + lane;
    const uint32_t prec_offset = 1u << (32 - (1 + 2 * kKsT));  // lwe-keyswitch-functions.cpp:119
    const uint32_t *my_cols = ring + cw * CW;
    int q = 0;
    bool failed = false;
    for (; q < i_count; q++) {
        if ((q & (kKsChunk - 1)) == 0) {
            // stage the next kKsChunk mask coefficients of the tile's samples, [coef][sample]
            __syncthreads();
            for (int e = tid; e < kKsTile * kKsChunk; e += kKsThreads) {
                const int g = e / kKsChunk, ii = e - g * kKsChunk;
                const int gg = tile * kKsTile + g;
                uint32_t v = 0;
                if (gg < count && q + ii < i_count) v = in[(size_t)gg * in_stride + i_begin + q + ii] + prec_offset;
                s_a[ii * L::sa_ld + g] = v;
            }
            __syncthreads();
        }
        const int s = q % L::stages;
        const bool ok = wait_bounded(bars + 8 * s, (q / L::stages) & 1, abort_flag, timeout_ns, err);
        const uint32_t abar = s_a[(q & (kKsChunk - 1)) * L::sa_ld + gl];
        const uint32_t *st = my_cols + s * L::stage_words;
#pragma unroll 2
        for (int j = 0; j < kKsT; j++) {
            // digit j from the top (lwe-keyswitch-functions.cpp:128-131); digit 0 reads the zero row
            const uint32_t d = (abar >> (30 - 2 * j)) & 3u;
            const int4 *row = reinterpret_cast<const int4 *>(st + (j * kKsBase + (int)d) * L::rs);
#pragma unroll
            for (int c4 = 0; c4 < CW / 4; c4++) {
                const int4 v = row[c4];
                acc[4 * c4 + 0] -= (uint32_t)v.x;
                acc[4 * c4 + 1] -= (uint32_t)v.y;
                acc[4 * c4 + 2] -= (uint32_t)v.z;
                acc[4 * c4 + 3] -= (uint32_t)v.w;
            }
        }
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        if (tid == 0 && !stall && issued < i_count) {
            issue(issued, s);
            issued++;
        }
    }
    if (failed) {
        // drain the copies still in flight before the CTA exits (each wait bounded)
        if (tid == 0) {
            volatile int32_t no_abort = 0;
            for (int r = q; r < issued; r++)
                wait_bounded(bars + 8 * (r % L::stages), (r / L::stages) & 1, &no_abort, timeout_ns, err);
        }
        return;
    }

    // transpose through shared memory so that each sample row is written with coalesced stores
    __syncthreads();
    uint32_t *stg = ring + warp * 32 * (CW + 1);
#pragma unroll
    for (int c = 0; c < CW; c++) stg[lane * (CW + 1) + c] = acc[c];
    __syncwarp();
    const int col0 = slice * L::slice + cw * CW;
    const int ncols = n + 1;
    for (int r = 0; r < 32; r++) {
        const int g = tile * kKsTile + gw * 32 + r;
        if (g >= count) break;
        uint32_t *o = out + (size_t)g * ncols;
        for (int c = lane; c < CW; c += 32) {
            const int col = col0 + c;
            if (col >= ncols) continue;
            uint32_t v = stg[r * (CW + 1) + c];
            // result = (0, b) - sum  (lwe-keyswitch-functions.cpp:233-237)
            if (col == n && kchunk == 0) v += in[(size_t)g * in_stride + kN];
            if (ksplit == 1) o[col] = v;
            else atomicAdd(o + col, v);
        }
    }
}

// ============================================================================================
// register-key kernel
// ============================================================================================
//
// One CTA of 8 warps per (8*G samples, block of 32*C output columns, range of input coefficients).
// Lane = column pair: lane l owns columns 64*p + 2*l + {0, 1}, p < C/2, so every shared load and
// global store of a warp touches consecutive words.  Per input coefficient i the block's key rows
// (t x 3 non-zero digits x 32*C columns) arrive in one bulk copy; per digit position j each lane
// loads its 3*C key words into registers once and applies them to the G samples of its warp.  A
// sample's digit is the same in every lane, so selecting the row is a warp-uniform branch and a
// zero digit costs no additions.  This lifts the one-word-per-subtraction shared-memory bound of
// the tiled kernel: each loaded word serves G samples.

template <int C, int G>
struct KsRegKey {
    static_assert(C % 2 == 0, "columns per lane come in pairs");
    static constexpr int block = 32 * C;                       // output columns per CTA
    static constexpr int rows = kKsT * (kKsBase - 1);          // non-zero digit rows per coefficient
    static constexpr int stage_words = rows * block;           // [j][digit 1..3][block]
    static constexpr int stage_bytes = 4 * stage_words;
    static constexpr int stages = stage_bytes <= 32768 ? 3 : 2;
    static constexpr int warps = 8;
    static constexpr int tile = warps * G;                     // samples per CTA
    static constexpr int sa_ld = tile + 1;
    static constexpr int ring_off = 128;                       // [0, 24): full barriers, [64]: abort flag
    static constexpr int sa_off = ring_off + stages * stage_bytes;
    static constexpr int smem_bytes = sa_off + 4 * kKsChunk * sa_ld;
    static_assert(stage_bytes % 16 == 0, "bulk copies need 16-byte sizes");
};

template <int C, int G>
__global__ void __launch_bounds__(256, 1)
    keyswitch_regkey_kernel(const int32_t *__restrict__ rows, const uint32_t *__restrict__ in, int in_stride,
                            uint32_t *__restrict__ out, int count, int n, int kN, int slices, int ksplit,
                            int chunk_len, uint64_t timeout_ns, int32_t *err, int stall) {
    using L = KsRegKey<C, G>;
    extern __shared__ __align__(128) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int kchunk = blockIdx.x % ksplit;
    const int unit = blockIdx.x / ksplit;
    const int slice = unit % slices, tile = unit / slices;
    const int i_begin = kchunk * chunk_len;
    const int i_count = min(kN, i_begin + chunk_len) - i_begin;

    const uint32_t bars = smem_addr(smem);
    volatile int32_t *abort_flag = reinterpret_cast<volatile int32_t *>(smem + 64);
    const uint32_t *ring = reinterpret_cast<const uint32_t *>(smem + L::ring_off);
    uint32_t *s_a = reinterpret_cast<uint32_t *>(smem + L::sa_off);
    if (tid == 0) {
        for (int s = 0; s < L::stages; s++) mbar_init(bars + 8 * s, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    const int32_t *src = rows + ((size_t)slice * kN + i_begin) * L::stage_words;
    auto issue = [&](int q, int s) {
        const uint32_t bar = bars + 8 * s;
        mbar_arrive_expect_tx(bar, L::stage_bytes);
        bulk_copy_g2s(smem_addr(ring + s * L::stage_words), src + (size_t)q * L::stage_words, L::stage_bytes, bar);
    };
    int issued = 0;  // meaningful in thread 0 only
    if (tid == 0 && !stall)  // stall: failure-detection test hook, no copy is ever issued
        for (; issued < L::stages && issued < i_count; issued++) issue(issued, issued);

    uint32_t acc[G][C];
#pragma unroll
    for (int s = 0; s < G; s++)
#pragma unroll
        for (int c = 0; c < C; c++) acc[s][c] = 0;
    const uint32_t prec_offset = 1u << (32 - (1 + 2 * kKsT));  // lwe-keyswitch-functions.cpp:119
    int q = 0;
    bool failed = false;
    for (; q < i_count; q++) {
        if ((q & (kKsChunk - 1)) == 0) {
            // stage the next kKsChunk mask coefficients of the tile's samples, [coef][sample]
            __syncthreads();
            for (int e = tid; e < L::tile * kKsChunk; e += 256) {
                const int g = e / kKsChunk, ii = e - g * kKsChunk;
                const int gg = tile * L::tile + g;
                uint32_t v = 0;
                if (gg < count && q + ii < i_count) v = in[(size_t)gg * in_stride + i_begin + q + ii] + prec_offset;
                s_a[ii * L::sa_ld + g] = v;
            }
            __syncthreads();
        }
        const int st_i = q % L::stages;
        const bool ok = wait_bounded(bars + 8 * st_i, (q / L::stages) & 1, abort_flag, timeout_ns, err);
        // every lane reads the same word; the OR over the warp returns it as a value the compiler
        // knows to be warp-uniform, so the digit arithmetic and the branches below can run on the
        // uniform datapath without convergence barriers
        uint32_t abar[G];
#pragma unroll
        for (int s = 0; s < G; s++)
            abar[s] = __reduce_or_sync(0xffffffffu, s_a[(q & (kKsChunk - 1)) * L::sa_ld + warp * G + s]);
        const uint32_t *stage = ring + st_i * L::stage_words + 2 * lane;
#pragma unroll 1
        for (int j = 0; j < kKsT; j++) {
            uint32_t k1[C], k2[C], k3[C];
            const uint32_t *rj = stage + j * (kKsBase - 1) * L::block;
#pragma unroll
            for (int p = 0; p < C / 2; p++) {
                const uint2 v1 = *reinterpret_cast<const uint2 *>(rj + 64 * p);
                const uint2 v2 = *reinterpret_cast<const uint2 *>(rj + L::block + 64 * p);
                const uint2 v3 = *reinterpret_cast<const uint2 *>(rj + 2 * L::block + 64 * p);
                k1[2 * p] = v1.x, k1[2 * p + 1] = v1.y;
                k2[2 * p] = v2.x, k2[2 * p + 1] = v2.y;
                k3[2 * p] = v3.x, k3[2 * p + 1] = v3.y;
            }
            const int sh = 30 - 2 * j;  // digit j from the top (lwe-keyswitch-functions.cpp:128-131)
#pragma unroll
            for (int s = 0; s < G; s++) {
                const uint32_t d = (abar[s] >> sh) & 3u;  // the same in every lane of the warp
                if (d == 1) {
#pragma unroll
                    for (int c = 0; c < C; c++) acc[s][c] -= k1[c];
                } else if (d == 2) {
#pragma unroll
                    for (int c = 0; c < C; c++) acc[s][c] -= k2[c];
                } else if (d == 3) {
#pragma unroll
                    for (int c = 0; c < C; c++) acc[s][c] -= k3[c];
                }
            }
        }
        if (__syncthreads_or(!ok)) {
            failed = true;
            break;
        }
        if (tid == 0 && !stall && issued < i_count) {
            issue(issued, st_i);
            issued++;
        }
    }
    if (failed) {
        // drain the copies still in flight before the CTA exits (each wait bounded)
        if (tid == 0) {
            volatile int32_t no_abort = 0;
            for (int r = q; r < issued; r++)
                wait_bounded(bars + 8 * (r % L::stages), (r / L::stages) & 1, &no_abort, timeout_ns, err);
        }
        return;
    }

    const int ncols = n + 1;
#pragma unroll
    for (int s = 0; s < G; s++) {
        const int g = tile * L::tile + warp * G + s;
        if (g >= count) break;
        uint32_t *o = out + (size_t)g * ncols;
        const uint32_t b = kchunk == 0 ? in[(size_t)g * in_stride + kN] : 0u;
#pragma unroll
        for (int c = 0; c < C; c++) {
            const int col = slice * L::block + 64 * (c >> 1) + 2 * lane + (c & 1);
            if (col >= ncols) continue;
            // result = (0, b) - sum  (lwe-keyswitch-functions.cpp:233-237)
            const uint32_t v = acc[s][c] + (col == n ? b : 0u);
            if (ksplit == 1) o[col] = v;
            else atomicAdd(o + col, v);
        }
    }
}

// ============================================================================================
// host side
// ============================================================================================

namespace {

bool tiled_params(const tfheb_params &p) { return p.ks_t == kKsT && (1 << p.ks_basebit) == kKsBase; }

// the compiled columns-per-warp choice with the least padding of n+1 (ties: the smaller)
int choose_cw(int n) {
    int best = 0, best_cols = 0;
    for (int cw : kKsCws) {
        const int slice = kKsColWarps * cw;
        const int cols = (n + 1 + slice - 1) / slice * slice;
        if (!best || cols < best_cols) best = cw, best_cols = cols;
    }
    return best;
}

template <int CW>
cudaError_t launch_tiled(const CloudKey &ck, int count, const int32_t *in, int in_stride, int32_t *out,
                         cudaStream_t s) {
    using L = KsTiled<CW>;
    const tfheb_params &p = ck.p;
    const int kN = p.k * p.N;
    cudaError_t e = cudaFuncSetAttribute(keyswitch_tiled_kernel<CW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         L::smem_bytes);
    if (e != cudaSuccess) return e;
    const int tiles = (count + kKsTile - 1) / kKsTile;
    const int units = tiles * ck.dksk.tile_slices;
    // split the coefficient range only when the units alone leave resident slots idle
    int ksplit = std::max(1, std::min(ck.dksk.tile_slots / units, kN / kKsChunk));
    int chunk_len = (kN + ksplit - 1) / ksplit;
    chunk_len = (chunk_len + kKsChunk - 1) / kKsChunk * kKsChunk;
    ksplit = (kN + chunk_len - 1) / chunk_len;
    if (ksplit > 1) {
        e = cudaMemsetAsync(out, 0, (size_t)count * (p.n + 1) * sizeof(int32_t), s);
        if (e != cudaSuccess) return e;
    }
    keyswitch_tiled_kernel<CW><<<units * ksplit, kKsThreads, L::smem_bytes, s>>>(
        ck.dksk.tiles, reinterpret_cast<const uint32_t *>(in), in_stride, reinterpret_cast<uint32_t *>(out), count,
        p.n, kN, ck.dksk.tile_slices, ksplit, chunk_len, ck.wait_timeout_ns, ck.d_err, ck.stall_producer);
    return cudaGetLastError();
}

// resident CTAs of the tiled kernel on the current device (all SMs)
template <int CW>
cudaError_t tiled_slots(int device, int *slots) {
    using L = KsTiled<CW>;
    cudaError_t e = cudaFuncSetAttribute(keyswitch_tiled_kernel<CW>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         L::smem_bytes);
    if (e != cudaSuccess) return e;
    int occ = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, keyswitch_tiled_kernel<CW>, kKsThreads, L::smem_bytes);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    *slots = std::max(occ, 1) * sms;
    return cudaSuccess;
}


// register-key instantiations: columns per lane C and samples per warp G
constexpr int kRkC[] = {10, 14};
int rk_samples_per_warp(int c) { return c == 10 ? 7 : 5; }

int choose_rk_c(int n) {
    int best = 0, best_cols = 0;
    for (int c : kRkC) {
        const int block = 32 * c;
        const int cols = (n + 1 + block - 1) / block * block;
        if (!best || cols < best_cols) best = c, best_cols = cols;
    }
    return best;
}

template <int C, int G>
cudaError_t regkey_slots(int device, int *slots) {
    using L = KsRegKey<C, G>;
    cudaError_t e = cudaFuncSetAttribute(keyswitch_regkey_kernel<C, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         L::smem_bytes);
    if (e != cudaSuccess) return e;
    int occ = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, keyswitch_regkey_kernel<C, G>, 256, L::smem_bytes);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    if (e != cudaSuccess) return e;
    *slots = std::max(occ, 1) * sms;
    return cudaSuccess;
}

template <int C, int G>
cudaError_t launch_regkey(const CloudKey &ck, int count, const int32_t *in, int in_stride, int32_t *out,
                          cudaStream_t s) {
    using L = KsRegKey<C, G>;
    const tfheb_params &p = ck.p;
    const int kN = p.k * p.N;
    cudaError_t e = cudaFuncSetAttribute(keyswitch_regkey_kernel<C, G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         L::smem_bytes);
    if (e != cudaSuccess) return e;
    const int tiles = (count + L::tile - 1) / L::tile;
    const int units = tiles * ck.dksk.rk_slices;
    // split the coefficient range only when the units alone leave resident slots idle
    int ksplit = std::max(1, std::min(ck.dksk.rk_slots / units, kN / kKsChunk));
    int chunk_len = (kN + ksplit - 1) / ksplit;
    chunk_len = (chunk_len + kKsChunk - 1) / kKsChunk * kKsChunk;
    ksplit = (kN + chunk_len - 1) / chunk_len;
    if (ksplit > 1) {
        e = cudaMemsetAsync(out, 0, (size_t)count * (p.n + 1) * sizeof(int32_t), s);
        if (e != cudaSuccess) return e;
    }
    keyswitch_regkey_kernel<C, G><<<units * ksplit, 256, L::smem_bytes, s>>>(
        ck.dksk.rk, reinterpret_cast<const uint32_t *>(in), in_stride, reinterpret_cast<uint32_t *>(out), count,
        p.n, kN, ck.dksk.rk_slices, ksplit, chunk_len, ck.wait_timeout_ns, ck.d_err, ck.stall_producer);
    return cudaGetLastError();
}

}  // namespace

cudaError_t upload_keyswitch_key(CloudKey &ck) {
    const tfheb_params &p = ck.p;
    DeviceKsk &d = ck.dksk;
    const int kN = p.k * p.N, t = p.ks_t, base = 1 << p.ks_basebit, ncols = p.n + 1;
    cudaError_t e;
    if (!d.rows) {
        d.stride = (ncols + 3) & ~3;
        const size_t rows = (size_t)kN * t * base;
        std::vector<int32_t> padded(rows * d.stride, 0);
        for (size_t r = 0; r < rows; r++)
            std::copy(&ck.ksk[r * ncols], &ck.ksk[r * ncols] + ncols, &padded[r * d.stride]);
        if ((e = cudaMalloc((void **)&d.rows, padded.size() * 4)) != cudaSuccess) return e;
        if ((e = cudaMemcpy(d.rows, padded.data(), padded.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess)
            return e;
    }
    if (!d.tiles && tiled_params(p)) {
        const int cw = choose_cw(p.n);
        const int slice = kKsColWarps * cw, rs = slice + 4;
        const int slices = (ncols + slice - 1) / slice;
        // [slice][i][j][digit 1..3][rs]; columns past n and the 4 pad words are zero
        std::vector<int32_t> tl((size_t)slices * kN * t * (base - 1) * rs, 0);
        for (int sl = 0; sl < slices; sl++)
            for (int i = 0; i < kN; i++)
                for (int j = 0; j < t; j++)
                    for (int h = 1; h < base; h++) {
                        const int32_t *srow = &ck.ksk[(((size_t)i * t + j) * base + h) * ncols];
                        int32_t *drow = &tl[((((size_t)sl * kN + i) * t + j) * (base - 1) + (h - 1)) * rs];
                        for (int c = 0; c < slice && sl * slice + c < ncols; c++) drow[c] = srow[sl * slice + c];
                    }
        if ((e = cudaMalloc((void **)&d.tiles, tl.size() * 4)) != cudaSuccess) return e;
        if ((e = cudaMemcpy(d.tiles, tl.data(), tl.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
        e = cw == 40 ? tiled_slots<40>(ck.device, &d.tile_slots) : tiled_slots<52>(ck.device, &d.tile_slots);
        if (e != cudaSuccess) return e;
        d.tile_cw = cw;
        d.tile_slices = slices;
    }
    if (!d.rk && tiled_params(p)) {
        const int c = choose_rk_c(p.n);
        const int block = 32 * c;
        const int slices = (ncols + block - 1) / block;
        // [slice][i][j][digit 1..3][block]; columns past n are zero
        std::vector<int32_t> rk((size_t)slices * kN * t * (base - 1) * block, 0);
        for (int sl = 0; sl < slices; sl++)
            for (int i = 0; i < kN; i++)
                for (int j = 0; j < t; j++)
                    for (int h = 1; h < base; h++) {
                        const int32_t *srow = &ck.ksk[(((size_t)i * t + j) * base + h) * ncols];
                        int32_t *drow = &rk[((((size_t)sl * kN + i) * t + j) * (base - 1) + (h - 1)) * block];
                        for (int col = 0; col < block && sl * block + col < ncols; col++)
                            drow[col] = srow[sl * block + col];
                    }
        if ((e = cudaMalloc((void **)&d.rk, rk.size() * 4)) != cudaSuccess) return e;
        if ((e = cudaMemcpy(d.rk, rk.data(), rk.size() * 4, cudaMemcpyHostToDevice)) != cudaSuccess) return e;
        e = c == 10 ? regkey_slots<10, 7>(ck.device, &d.rk_slots) : regkey_slots<14, 5>(ck.device, &d.rk_slots);
        if (e != cudaSuccess) return e;
        d.rk_c = c;
        d.rk_slices = slices;
    }
    return upload_keyswitch_key_mma(ck);
}

void free_keyswitch_key(DeviceKsk &d) {
    if (d.rows) cudaFree(d.rows);
    if (d.tiles) cudaFree(d.tiles);
    if (d.rk) cudaFree(d.rk);
    if (d.mma) cudaFree(d.mma);
    d = DeviceKsk{};
}

cudaError_t launch_keyswitch(const CloudKey &ck, int count, const int32_t *in, int in_stride, int32_t *out,
                             cudaStream_t s) {
    if (count <= 0) return cudaSuccess;
    const tfheb_params &p = ck.p;
    // default: the tensor-core kernel wherever it is built (t = 8, basebit = 2), at every batch size
    // (measured per 4096 / 1036 / 256 / 1 samples: 0.305 / 0.114 / 0.044 / 0.035 ms, against 1.82 /
    // 0.578 / 0.225 / 0.077 ms for the register-key and 2.89 / 0.738 / 0.196 / 0.049 ms for the
    // tiled kernel); otherwise the one-CTA-per-sample kernel
    if ((ck.ks_kernel == 4 || ck.ks_kernel == 0) && ck.dksk.mma_groups != 0)
        return launch_keyswitch_mma(ck, count, in, in_stride, out, s);
    const bool regkey = ck.ks_kernel == 3;
    if (regkey && ck.dksk.rk_c != 0) {
        switch (ck.dksk.rk_c) {
            case 10: return launch_regkey<10, 7>(ck, count, in, in_stride, out, s);
            case 14: return launch_regkey<14, 5>(ck, count, in, in_stride, out, s);
            default: return cudaErrorInvalidValue;
        }
    }
    const bool tiled = ck.dksk.tile_cw != 0 && ck.ks_kernel != 1;
    if (tiled) {
        switch (ck.dksk.tile_cw) {
            case 40: return launch_tiled<40>(ck, count, in, in_stride, out, s);
            case 52: return launch_tiled<52>(ck, count, in, in_stride, out, s);
            default: return cudaErrorInvalidValue;
        }
    }
    const int kN = p.k * p.N;
    const int threads = ((ck.dksk.stride / 4 + 31) / 32) * 32;
    if (threads > 256) return cudaErrorInvalidValue;
    keyswitch_gate_kernel<<<count, threads, sizeof(uint32_t) * kN, s>>>(
        ck.dksk.rows, ck.dksk.stride, reinterpret_cast<const uint32_t *>(in), in_stride,
        reinterpret_cast<uint32_t *>(out), p.n, kN, p.ks_t, p.ks_basebit);
    return cudaGetLastError();
}

}  // namespace tfheb
