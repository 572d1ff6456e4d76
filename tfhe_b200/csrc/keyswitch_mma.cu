// keyswitch_mma.cu -- the LWE keyswitch (lweKeySwitch, lwe-keyswitch-functions.cpp:228-238, through
// lweKeySwitchTranslate_fromArray, :111-136) on the tensor cores, for t = 8 digits of 2 bits.
//
// The keyswitch subtracts, for every mask coefficient i and digit position j, the key sample
// ks[i][j][h] that digit j of abar_i = a_i + 2^(32-(1+2t)) selects; h = 0 is skipped.  That is a
// product of a one-hot matrix with the key:
//     A[s][(i, j, h)] = (digit j of sample s's abar_i == h),   B[(i, j, h)][col] = ks[i][j][h][col]
// with the h = 0 rows of B zero.  Modulo 2^32 the key splits into four byte planes,
// B = sum_p 2^(8p) B_p, and each A x B_p is an exact product of u8 matrices with s32 sums: an entry
// adds t = 8 bytes per coefficient, at most kN * 8 * 255 < 2^23.  So
//     out[s][col] = (col == n ? b_s : 0) - sum_p 2^(8p) (A x B_p)[s][col]   (mod 2^32),
// the reference's result bit for bit.
//
// Tiling.  A CTA takes 256 samples (two accumulators of M = 128 rows) x 64 output columns, whose
// four byte planes make N = 256 (plane p of column c at n = 64 p + c).  K runs over the
// coefficients, 32 bytes each (8 digit positions x 4 digit values, byte 4j + h), so one
// tcgen05.mma.kind::i8 of M 128, N 256, K 32 per coefficient and accumulator; the two accumulators
// take all 512 TMEM columns.  A CTA can be given a range of the coefficients (the partial sums then
// meet in the output through atomic adds, exact modulo 2^32), so that small batches fill the GPU.
//
// Roles (320 threads):
//   warps 0-7  one sample row each: write the row's one-hot A bytes (two 16-byte stores per
//              coefficient, from the abar word) into the stage, then, after the last product, read
//              the row's accumulators from TMEM, combine the planes and store the 64 columns;
//   warp 8     lane 0 streams B: one bulk copy per stage from the device key, laid out offline in
//              the exact shared-memory image the descriptors describe;
//   warp 9     lane 0 issues the products and commits each stage back to the producers.
// Operands use the no-swizzle K-major layout: core matrices of 8 rows x 16 bytes, the two 16-byte K
// halves of a row 128 bytes apart, 8-row groups 256 bytes apart.
// Every mbarrier wait is bounded (async_copy.cuh).  After a wait runs out, each role stops, the copy
// issuer waits for its copies in flight, the issuing thread waits for its products, and warp 0
// frees the TMEM columns after the final barrier.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <vector>

#include "async_copy.cuh"
#include "internal.h"
#include "tmem.cuh"

namespace tfheb {

namespace {

constexpr int kKmT = 8;                                   // digit positions
constexpr int kKmRows = 128;                              // samples per accumulator (M)
constexpr int kKmHalves = 2;                              // accumulators per CTA
constexpr int kKmTile = kKmRows * kKmHalves;              // samples per CTA
constexpr int kKmCols = 64;                               // output columns per CTA
constexpr int kKmN = 4 * kKmCols;                         // byte planes x columns (N)
constexpr int kKmKS = 2;                                  // coefficients per pipeline stage
constexpr int kKmStages = 6;
constexpr int kKmABytes = kKmRows * 32;                   // one accumulator's A for one coefficient
constexpr int kKmBBytes = kKmN * 32;                      // B for one coefficient (8 KB)
constexpr int kKmStageA = kKmHalves * kKmKS * kKmABytes;  // 16 KB
constexpr int kKmStageB = kKmKS * kKmBBytes;              // 16 KB
constexpr int kKmStageBytes = kKmStageA + kKmStageB;
constexpr int kKmBarOff = kKmStages * kKmStageBytes;      // 192 KB of stages
constexpr int kKmMiscOff = kKmBarOff + (3 * kKmStages + 1) * 8;
constexpr int kKmSmem = kKmMiscOff + 16;
constexpr int kKmProducers = kKmTile;                     // one thread per sample row
constexpr int kKmThreads = kKmProducers + 64;
constexpr int kKmGroup = 8;                               // coefficients whose inputs a row loads at once
constexpr int kKmStageLd = kKmCols + 1;                   // staging row length (words) of the epilogue
constexpr uint32_t kKmTmemCols = kKmHalves * kKmN;        // 512

static_assert(kKmSmem <= 227 * 1024, "shared memory");
static_assert(kKmTile * kKmStageLd * 4 <= kKmBarOff, "the epilogue staging reuses the stages");
static_assert(kKmGroup % kKmKS == 0, "whole stages per input group");
static_assert(kKmTmemCols == 512, "two accumulators of N columns fill TMEM");

// byte offset of (row, k-byte) in an operand of the no-swizzle K-major layout
__host__ __device__ constexpr uint32_t km_offset(int row, int kb) {
    return (uint32_t)((row >> 3) * 256 + (kb >> 4) * 128 + (row & 7) * 16 + (kb & 15));
}

__global__ void __launch_bounds__(kKmThreads, 1)
    keyswitch_mma_kernel(const uint8_t *__restrict__ bkey, const uint32_t *__restrict__ in, int in_stride,
                         uint32_t *__restrict__ out, int count, int n, int kN, int groups, int ksplit, int chunk_len,
                         uint64_t timeout_ns, int32_t *err, int stall) {
    extern __shared__ __align__(1024) unsigned char smem[];
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int kchunk = blockIdx.x % ksplit;
    const int g = (blockIdx.x / ksplit) % groups;
    const int tile = blockIdx.x / (ksplit * groups);
    const int i_begin = kchunk * chunk_len;
    const int nq = chunk_len / kKmKS;  // pipeline stages of this CTA

    const uint32_t sbase = smem_addr(smem);
    const uint32_t full_a = sbase + kKmBarOff, full_b = full_a + 8 * kKmStages, empty = full_b + 8 * kKmStages;
    const uint32_t done = empty + 8 * kKmStages;
    uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(smem + kKmMiscOff);
    volatile int32_t *abort_flag = reinterpret_cast<volatile int32_t *>(smem + kKmMiscOff + 4);
    if (tid == 0) {
        for (int s = 0; s < kKmStages; s++) {
            mbar_init(full_a + 8 * s, kKmProducers);
            mbar_init(full_b + 8 * s, 1);
            mbar_init(empty + 8 * s, 1);
        }
        mbar_init(done, 1);
        *abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) tmem_alloc(smem_addr(tmem_slot), kKmTmemCols);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const uint32_t tmem_base = *tmem_slot;

    if (tid < kKmProducers) {
        // ---- one-hot rows ----
        const int h = tid / kKmRows, rr = tid % kKmRows;
        const int sample = tile * kKmTile + tid;
        const bool live = sample < count;
        const uint32_t *src = in + (size_t)(live ? sample : 0) * in_stride + i_begin;
        const uint32_t prec_offset = 1u << (32 - (1 + 2 * kKmT));  // lwe-keyswitch-functions.cpp:119
        unsigned char *a_row = smem + h * (kKmKS * kKmABytes) + km_offset(rr, 0);
        uint32_t cur[kKmGroup], nxt[kKmGroup];
#pragma unroll
        for (int e = 0; e < kKmGroup; e++) cur[e] = live ? __ldg(src + e) : 0u;
        bool ok = true;
        for (int q0 = 0; q0 < nq && ok; q0 += kKmGroup / kKmKS) {
            const int inext = (q0 + kKmGroup / kKmKS) * kKmKS;
#pragma unroll
            for (int e = 0; e < kKmGroup; e++) nxt[e] = (live && inext < chunk_len) ? __ldg(src + inext + e) : 0u;
#pragma unroll
            for (int qq = 0; qq < kKmGroup / kKmKS; qq++) {
                const int q = q0 + qq, s = q % kKmStages;
                if (q >= kKmStages && !wait_bounded(empty + 8 * s, ((q / kKmStages) - 1) & 1, abort_flag, timeout_ns, err)) {
                    ok = false;
                    break;
                }
                unsigned char *a = a_row + s * kKmStageBytes;
#pragma unroll
                for (int k = 0; k < kKmKS; k++) {
                    const uint32_t x = cur[qq * kKmKS + k] + prec_offset;
                    uint32_t w[kKmT];
#pragma unroll
                    for (int j = 0; j < kKmT; j++)  // byte 4j + digit j, digit j from the top (:128-131)
                        w[j] = live ? 1u << ((x >> (27 - 2 * j)) & 24u) : 0u;
                    *reinterpret_cast<uint4 *>(a + k * kKmABytes) = make_uint4(w[0], w[1], w[2], w[3]);
                    *reinterpret_cast<uint4 *>(a + k * kKmABytes + 128) = make_uint4(w[4], w[5], w[6], w[7]);
                }
                fence_proxy_async_smem();
                mbar_arrive(full_a + 8 * s);
            }
#pragma unroll
            for (int e = 0; e < kKmGroup; e++) cur[e] = nxt[e];
        }
    } else if (warp == kKmProducers / 32 && lane == 0) {
        // ---- key stream ----
        const uint8_t *bsrc = bkey + ((size_t)g * kN + i_begin) * kKmBBytes;
        int issued = 0;
        if (!stall) {  // stall: failure-detection test hook, no copy is ever issued
            for (int q = 0; q < nq; q++) {
                const int s = q % kKmStages;
                if (q >= kKmStages && !wait_bounded(empty + 8 * s, ((q / kKmStages) - 1) & 1, abort_flag, timeout_ns, err))
                    break;
                mbar_arrive_expect_tx(full_b + 8 * s, kKmStageB);
                bulk_copy_g2s(sbase + s * kKmStageBytes + kKmStageA, bsrc + (size_t)q * kKmStageB, kKmStageB,
                              full_b + 8 * s);
                issued++;
            }
        }
        // copies still in flight land before the CTA exits (each wait bounded)
        volatile int32_t no_abort = 0;
        for (int q = std::max(0, issued - kKmStages); q < issued; q++)
            wait_bounded(full_b + 8 * (q % kKmStages), (q / kKmStages) & 1, &no_abort, timeout_ns, err);
    } else if (warp == kKmProducers / 32 + 1 && lane == 0) {
        // ---- products ----
        const uint32_t idesc = umma_idesc_u8_s32(kKmRows, kKmN);
        for (int q = 0; q < nq; q++) {
            const int s = q % kKmStages, par = (q / kKmStages) & 1;
            if (!wait_bounded(full_a + 8 * s, par, abort_flag, timeout_ns, err) ||
                !wait_bounded(full_b + 8 * s, par, abort_flag, timeout_ns, err))
                break;
            tmem_fence_after_sync();
            const uint32_t stage = sbase + s * kKmStageBytes;
#pragma unroll
            for (int k = 0; k < kKmKS; k++) {
                const uint64_t bdesc = umma_desc_kmajor(stage + kKmStageA + k * kKmBBytes, 128, 256);
#pragma unroll
                for (int hh = 0; hh < kKmHalves; hh++) {
                    const uint64_t adesc = umma_desc_kmajor(stage + (hh * kKmKS + k) * kKmABytes, 128, 256);
                    umma_u8(tmem_base + (uint32_t)(hh * kKmN), adesc, bdesc, idesc, (q | k) != 0);
                }
            }
            umma_commit(empty + 8 * s);
        }
        umma_commit(done);
        // the products issued so far complete before the CTA exits (the wait is bounded)
        volatile int32_t no_abort = 0;
        wait_bounded(done, 0, &no_abort, timeout_ns, err);
    }

    if (tid < kKmProducers) {
        // ---- epilogue: accumulators -> columns ----
        bool ok = wait_bounded(done, 0, abort_flag, timeout_ns, err);
        ok = __all_sync(0xffffffffu, ok);  // tcgen05.ld is warp-collective
        if (ok) {
            tmem_fence_after_sync();
            const int h = warp / 4, quad = warp % 4;  // row tid = 128 h + 32 quad + lane
            const uint32_t t_row = tmem_base + ((uint32_t)(quad * 32) << 16) + (uint32_t)(h * kKmN);
            uint32_t *stg = reinterpret_cast<uint32_t *>(smem);
#pragma unroll 1
            for (int c0 = 0; c0 < kKmCols; c0 += 16) {
                uint32_t p0[16], p1[16], p2[16], p3[16];
                tmem_ld16(t_row + c0, p0);
                tmem_ld16(t_row + kKmCols + c0, p1);
                tmem_ld16(t_row + 2 * kKmCols + c0, p2);
                tmem_ld16(t_row + 3 * kKmCols + c0, p3);
                tmem_wait_ld16(p0);
                tmem_wait_ld16(p1);
                tmem_wait_ld16(p2);
                tmem_wait_ld16(p3);
#pragma unroll
                for (int e = 0; e < 16; e++)
                    stg[tid * kKmStageLd + c0 + e] = p0[e] + (p1[e] << 8) + (p2[e] << 16) + (p3[e] << 24);
            }
            __syncwarp();
            // the warp stores its own 32 rows, a row's 64 columns per pass (coalesced)
            const int ncols = n + 1;
            for (int r = 0; r < 32; r++) {
                const int row = warp * 32 + r, sample = tile * kKmTile + row;
                if (sample >= count) break;
                const uint32_t b = kchunk == 0 ? in[(size_t)sample * in_stride + kN] : 0u;
                uint32_t *o = out + (size_t)sample * ncols;
#pragma unroll
                for (int half = 0; half < 2; half++) {
                    const int c = half * 32 + lane, col = g * kKmCols + c;
                    if (col >= ncols) continue;
                    // result = (0, b) - sum  (lwe-keyswitch-functions.cpp:233-237)
                    const uint32_t v = (col == n ? b : 0u) - stg[row * kKmStageLd + c];
                    if (ksplit == 1) o[col] = v;
                    else atomicAdd(o + col, v);
                }
            }
        }
    }

    tmem_fence_before_sync();
    __syncthreads();
    if (warp == 0) {
        tmem_fence_after_sync();
        tmem_free(tmem_base, kKmTmemCols);
    }
}

}  // namespace

// ============================================================================================
// host side
// ============================================================================================

int km_groups(const tfheb_params &p) { return (p.n + 1 + kKmCols - 1) / kKmCols; }

// The key in the shared-memory image of the B operand: [group][coefficient i][8 KB], byte plane p of
// ks[i][j][h][64 g + c] at (row 64 p + c, k-byte 4 j + h); h = 0 and columns past n stay zero.
cudaError_t upload_keyswitch_key_mma(CloudKey &ck) {
    const tfheb_params &p = ck.p;
    DeviceKsk &d = ck.dksk;
    if (d.mma || p.ks_t != kKmT || p.ks_basebit != 2) return cudaSuccess;
    const int kN = p.k * p.N, t = p.ks_t, base = 1 << p.ks_basebit, ncols = p.n + 1;
    const int groups = km_groups(p);
    std::vector<uint8_t> img((size_t)groups * kN * kKmBBytes, 0);
    for (int g = 0; g < groups; g++)
        for (int i = 0; i < kN; i++) {
            uint8_t *blk = &img[((size_t)g * kN + i) * kKmBBytes];
            for (int j = 0; j < t; j++)
                for (int h = 1; h < base; h++) {
                    const int32_t *srow = &ck.ksk[(((size_t)i * t + j) * base + h) * ncols];
                    const int kb = j * base + h;
                    for (int c = 0; c < kKmCols && g * kKmCols + c < ncols; c++) {
                        const uint32_t v = (uint32_t)srow[g * kKmCols + c];
                        for (int pl = 0; pl < 4; pl++) blk[km_offset(pl * kKmCols + c, kb)] = (uint8_t)(v >> (8 * pl));
                    }
                }
        }
    cudaError_t e;
    if ((e = cudaMalloc((void **)&d.mma, img.size())) != cudaSuccess) return e;
    if ((e = cudaMemcpy(d.mma, img.data(), img.size(), cudaMemcpyHostToDevice)) != cudaSuccess) return e;
    if ((e = cudaFuncSetAttribute(keyswitch_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kKmSmem)) !=
        cudaSuccess)
        return e;
    d.mma_groups = groups;
    return cudaSuccess;
}

// Coefficient split: the CTA count (tiles x groups x split) is rounded up to whole waves of one CTA
// per SM, and each CTA pays a fixed cost (TMEM allocation, pipeline fill, epilogue) of about
// kKmUnitCost coefficients; the split with the least modelled time wins.
constexpr int kKmUnitCost = 32;

cudaError_t launch_keyswitch_mma(const CloudKey &ck, int count, const int32_t *in, int in_stride, int32_t *out,
                                 cudaStream_t s) {
    const tfheb_params &p = ck.p;
    const int kN = p.k * p.N;
    if (!ck.dksk.mma) return cudaErrorInvalidValue;
    int sms = 0;
    cudaError_t e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ck.device);
    if (e != cudaSuccess) return e;
    const int groups = ck.dksk.mma_groups;
    const long units = (long)((count + kKmTile - 1) / kKmTile) * groups;
    int ksplit = 1;
    long best = -1;
    for (int ks = 1; ks <= 16; ks *= 2) {
        if (kN % ks || (kN / ks) % kKmGroup) break;
        const long waves = (units * ks + sms - 1) / sms;
        const long cost = waves * (kN / ks + kKmUnitCost);
        if (best < 0 || cost < best) best = cost, ksplit = ks;
    }
    const int chunk_len = kN / ksplit;
    if (ksplit > 1 && (e = cudaMemsetAsync(out, 0, (size_t)count * (p.n + 1) * sizeof(int32_t), s)) != cudaSuccess)
        return e;
    keyswitch_mma_kernel<<<(unsigned)(units * ksplit), kKmThreads, kKmSmem, s>>>(
        ck.dksk.mma, reinterpret_cast<const uint32_t *>(in), in_stride, reinterpret_cast<uint32_t *>(out), count, p.n,
        kN, groups, ksplit, chunk_len, ck.wait_timeout_ns, ck.d_err, ck.stall_producer);
    return cudaGetLastError();
}

}  // namespace tfheb
