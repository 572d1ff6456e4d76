// netlist.cu -- levelled evaluation of a gate netlist on the GPU, replayed as a CUDA graph.
//
// The reference evaluates circuits one gate call at a time (e.g. test-long-run.cpp:61-185,
// test-addition-boot.cpp); here the whole circuit is scheduled at creation:
//   * each gate gets a level: the earliest is 1 + the deepest level among its inputs (primary inputs
//     are level 0); gates with slack then move later to fill blind-rotation waves (pack_levels),
//     keeping the number of levels at the critical path length;
//   * gates are renumbered level by level into an internal wire array, bootstrapped gates first in
//     each level, so a level's outputs are one contiguous block of rows;
//   * per level, one launch sequence covers all its gates whatever their types: a prologue that reads
//     operands by wire row, one blind-rotation launch over all bootstraps of the level (two per MUX),
//     extraction, keyswitch straight into the level's output rows, and a copy/negate kernel for
//     bootstrap-free NOT/COPY gates;
//   * descriptors of all levels are uploaded once; the first run on a (precision, wire array) pair
//     captures the level sequence into a CUDA graph, later runs replay it with one launch.
// The same level launch sequence serves two more entry points: a batch of mixed gate types over
// caller-given wire rows (tfheb_gate_batch_mixed_device), and a netlist sharded across several keys
// and GPUs (tfheb_netlist_multi_*), whose shards exchange each level's outputs by peer copies.
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "internal.h"

namespace tfheb {
namespace {

struct BootDescRows {
    int32_t xrow, yrow;  // operand rows in the internal wire array
    int32_t cst;
    int8_t sa, sb;
    int16_t pad;
};

struct UnaryDesc {
    int32_t src, dst;
    int32_t negate;
};

__device__ __forceinline__ int32_t modswitch_rows(uint32_t phase, uint64_t interv) {
    const uint64_t phase64 = ((uint64_t)phase << 32) + (interv >> 1);
    return (int32_t)(phase64 / interv);
}

// gate prologue with operands addressed by wire row (boot-gates.cpp:34-370, numeric-functions.cpp:59-65)
__global__ void prologue_rows_kernel(const BootDescRows *__restrict__ desc, const uint32_t *__restrict__ wires, int n,
                                     uint64_t interv, int32_t *__restrict__ bara, int bara_stride) {
    const BootDescRows d = desc[blockIdx.x];
    const uint32_t *x = wires + (size_t)d.xrow * (n + 1);
    const uint32_t *y = wires + (size_t)d.yrow * (n + 1);
    int32_t *out = bara + (size_t)blockIdx.x * bara_stride;
    for (int i = threadIdx.x; i <= n; i += blockDim.x) {
        uint32_t v = (uint32_t)(int32_t)d.sa * x[i] + (uint32_t)(int32_t)d.sb * y[i];
        if (i == n) v += (uint32_t)d.cst;
        out[i] = modswitch_rows(v, interv);
    }
}

// bootstrap-free gates: NOT negates, COPY copies (boot-gates.cpp:164-178); rows of `from` -> rows of `to`
__global__ void unary_rows_kernel(const UnaryDesc *__restrict__ desc, const uint32_t *from, uint32_t *to, int n) {
    const UnaryDesc d = desc[blockIdx.x];
    const uint32_t *src = from + (size_t)d.src * (n + 1);
    uint32_t *dst = to + (size_t)d.dst * (n + 1);
    for (int i = threadIdx.x; i <= n; i += blockDim.x) dst[i] = d.negate ? 0u - src[i] : src[i];
}

// rows of `src` -> rows perm[r] of `dst` (and the identity copy of the primary inputs)
__global__ void permute_rows_kernel(const int32_t *__restrict__ perm, const uint32_t *__restrict__ src,
                                    uint32_t *__restrict__ dst, int n, int src_offset) {
    const int r = blockIdx.x;
    const uint32_t *s = src + (size_t)(src_offset + r) * (n + 1);
    uint32_t *d = dst + (size_t)perm[r] * (n + 1);
    for (int i = threadIdx.x; i <= n; i += blockDim.x) d[i] = s[i];
}

struct Level {
    int boot_off, boots;     // into the concatenated BootDescRows
    int gate_off, gates;     // bootstrapped gates: into the concatenated GateDesc
    int unary_off, unaries;  // into the concatenated UnaryDesc
    int out_row;             // first internal row of the bootstrapped outputs (rows out_row .. +gates)
};

}  // namespace
}  // namespace tfheb

namespace tfheb {
namespace {
// One level schedule of a netlist: levels, their descriptors and the internal row order.  Each
// precision has its own, packed for the wave of that precision's blind-rotation variant.
struct Schedule {
    std::vector<Level> levels;
    int max_boots = 0, max_gates = 0;
    BootDescRows *d_boot = nullptr;
    GateDesc *d_gate = nullptr;
    UnaryDesc *d_unary = nullptr;
    int32_t *d_out_perm = nullptr;  // internal gate row (minus num_inputs) -> user row
    int graph_kernels = 0;          // kernels replayed by one graph launch
    void release() {
        cudaFree(d_boot);
        cudaFree(d_gate);
        cudaFree(d_unary);
        cudaFree(d_out_perm);
    }
};
}  // namespace
}  // namespace tfheb

struct tfheb_netlist {
    tfheb_cloud_key *ck = nullptr;
    int num_inputs = 0, num_gates = 0;
    tfheb::Schedule sched[2];       // [TFHEB_FP64], [TFHEB_SPLIT_FP32]
    // device state shared by both schedules
    int32_t *d_wires = nullptr;     // internal wire array [num_inputs + num_gates][n+1]
    int32_t *d_bara = nullptr, *d_acc = nullptr, *d_ksin = nullptr;
    std::map<std::pair<int, const int32_t *>, cudaGraphExec_t> graphs;
    std::map<std::pair<int, const int32_t *>, cudaGraph_t> graph_defs;
    // runs may come on different streams: each waits on the device for the previous run to finish
    // with the shared state above, then marks its own end
    cudaEvent_t run_done = nullptr;
};

// A netlist sharded across cloud keys on several devices: one schedule per key and precision
// (build_schedule's shards), a full wire array per key, and after every level an all-gather of the
// shards' outputs by peer copies.
struct tfheb_netlist_multi {
    std::vector<tfheb_cloud_key *> cks;
    int num_inputs = 0, num_gates = 0, nlev = 0;
    struct Shard {
        tfheb::Schedule sched[2];
        int32_t *d_wires = nullptr, *d_bara = nullptr, *d_acc = nullptr, *d_ksin = nullptr;
        cudaEvent_t copied = nullptr;  // recorded on the key's stream after its copies of a level
    };
    std::vector<Shard> shards;
    int32_t *d_user = nullptr;  // on key 0's device: the gates' rows in user order
};

using namespace tfheb;

namespace {

tfheb_status nl_fail(const std::string &msg, tfheb_status st = TFHEB_ERR_INVALID) {
    set_error(msg);
    return st;
}

// Scratch of one schedule on one device.
struct LevelScratch {
    int32_t *wires, *bara, *acc, *ksin;
};

// One level of schedule `sc` on stream s: prologue, blind rotation, extraction and keyswitch of its
// bootstrapped gates (outputs to rows L.out_row..), then its NOT/COPY gates.
cudaError_t enqueue_level(const Schedule &sc, const Level &L, CloudKey &ck, int precision, const LevelScratch &w,
                          cudaStream_t s, int &launches) {
    const tfheb_params &p = ck.p;
    const int n1 = p.n + 1, kN1 = p.k * p.N + 1, bs = bara_stride_for(p);
    const uint64_t interv = ((UINT64_C(1) << 63) / (uint64_t)(2 * p.N)) * 2;
    cudaError_t e = cudaSuccess;
    if (L.boots > 0) {
        prologue_rows_kernel<<<L.boots, 256, 0, s>>>(sc.d_boot + L.boot_off, reinterpret_cast<const uint32_t *>(w.wires),
                                                     p.n, interv, w.bara, bs);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        e = launch_blind_rotate(p, precision, ck.dbsk[precision], w.bara, bs, L.boots, p.n, modswitch_to_torus32(1, 8),
                                nullptr, w.acc, s, ck.d_err, ck.stall_producer, ck.wait_timeout_ns,
                                ck.br[precision]);
        if (e != cudaSuccess) return e;
        e = launch_extract(p, sc.d_gate + L.gate_off, L.gates, w.acc, w.ksin, kN1, s);
        if (e != cudaSuccess) return e;
        e = launch_keyswitch(ck, L.gates, w.ksin, kN1, w.wires + (size_t)L.out_row * n1, s);
        if (e != cudaSuccess) return e;
        launches += 4;
    }
    if (L.unaries > 0) {
        unary_rows_kernel<<<L.unaries, 256, 0, s>>>(sc.d_unary + L.unary_off, reinterpret_cast<const uint32_t *>(w.wires),
                                                     reinterpret_cast<uint32_t *>(w.wires), p.n);
        e = cudaGetLastError();
        launches += 1;
    }
    return e;
}

// Enqueues the whole level sequence on stream s (also used inside stream capture).
cudaError_t enqueue_netlist(tfheb_netlist *nl, CloudKey &ck, int precision, int32_t *user_wires, cudaStream_t s,
                            int *kernels) {
    const tfheb_params &p = ck.p;
    const int n1 = p.n + 1;
    cudaError_t e = cudaMemcpyAsync(nl->d_wires, user_wires, (size_t)nl->num_inputs * n1 * 4,
                                    cudaMemcpyDeviceToDevice, s);
    int launches = 0;
    const Schedule &sc = nl->sched[precision];
    const LevelScratch w{nl->d_wires, nl->d_bara, nl->d_acc, nl->d_ksin};
    for (const Level &L : sc.levels) {
        if (e != cudaSuccess) break;
        e = enqueue_level(sc, L, ck, precision, w, s, launches);
    }
    if (e == cudaSuccess && nl->num_gates > 0) {
        permute_rows_kernel<<<nl->num_gates, 256, 0, s>>>(sc.d_out_perm, reinterpret_cast<const uint32_t *>(nl->d_wires),
                                                          reinterpret_cast<uint32_t *>(user_wires), p.n, nl->num_inputs);
        e = cudaGetLastError();
        launches += 1;
    }
    *kernels = launches;
    return e;
}

// Bootstraps one blind-rotation launch runs per wave: SMs x bootstraps per CTA of the key's current
// variant for `precision`.
int wave_bootstraps(const CloudKey &ck, int precision) {
    int sms = 0, G[16] = {0}, D[16] = {0};
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, ck.device);
    const int nv = br_variants(ck.p.N, ck.p.l, precision, G, D, 16);
    const int v = ck.br[precision].tuned;
    return std::max(1, sms) * (nv > 0 && v < nv ? G[v] : 1);
}

// Level assignment that fills blind-rotation waves.  `level` holds each gate's earliest level
// (1 + its deepest input) on entry.  Every gate gets a deadline, its latest level that keeps the
// number of levels at nlev (1 below the earliest deadline among its consumers; nlev without
// consumers).  Level s then takes every ready gate whose deadline is s, and tops the level up with
// other ready gates, earliest deadline first, while its bootstraps stay within the waves the
// mandatory gates already start (a multiple of `wave`).  A gate is ready once all its inputs sit on
// earlier levels, so the evaluation order stays valid; NOT/COPY gates (no bootstrap) go on the
// first level where they are ready.
void pack_levels(int num_inputs, int num_gates, const int32_t *gates, const int32_t *in_a, const int32_t *in_b,
                 const int32_t *in_c, int nlev, int wave, std::vector<int> &level) {
    if (num_gates == 0 || wave <= 1) return;
    const int32_t *ins[3] = {in_a, in_b, in_c};
    auto nin = [&](int g) { return gates[g] == TFHEB_MUX ? 3 : (gates[g] >= TFHEB_NOT ? 1 : 2); };
    auto boots = [&](int g) { return gates[g] == TFHEB_MUX ? 2 : (gates[g] >= TFHEB_NOT ? 0 : 1); };
    // deadlines, consumers first (a gate only reads earlier wires)
    std::vector<int> deadline(num_gates, nlev);
    for (int g = num_gates - 1; g >= 0; g--)
        for (int k = 0; k < nin(g); k++) {
            const int src = ins[k][g] - num_inputs;
            if (src >= 0) deadline[src] = std::min(deadline[src], deadline[g] - 1);
        }
    // consumer lists and unscheduled-input counts
    std::vector<int> cons_off(num_gates + 1, 0), waiting(num_gates, 0);
    for (int g = 0; g < num_gates; g++)
        for (int k = 0; k < nin(g); k++) {
            const int src = ins[k][g] - num_inputs;
            if (src >= 0) cons_off[src + 1]++, waiting[g]++;
        }
    for (int g = 0; g < num_gates; g++) cons_off[g + 1] += cons_off[g];
    std::vector<int> cons(cons_off[num_gates]), fill(cons_off.begin(), cons_off.end() - 1);
    for (int g = 0; g < num_gates; g++)
        for (int k = 0; k < nin(g); k++) {
            const int src = ins[k][g] - num_inputs;
            if (src >= 0) cons[fill[src]++] = g;
        }
    // ready gates bucketed by deadline; unary gates in their own list
    std::vector<std::vector<int>> bucket(nlev + 2);
    std::vector<size_t> head(nlev + 2, 0);
    std::vector<int> unary_ready;
    auto make_ready = [&](int g) {
        if (boots(g) == 0) unary_ready.push_back(g);
        else bucket[deadline[g]].push_back(g);
    };
    for (int g = 0; g < num_gates; g++)
        if (waiting[g] == 0) make_ready(g);
    std::vector<int> placed;
    for (int s = 1; s <= nlev; s++) {
        placed.clear();
        std::vector<int> un;
        un.swap(unary_ready);
        for (int g : un) placed.push_back(g);
        int used = 0;
        for (; head[s] < bucket[s].size(); head[s]++) {  // mandatory: deadline s
            const int g = bucket[s][head[s]];
            placed.push_back(g);
            used += boots(g);
        }
        const int cap = (std::max(used, 1) + wave - 1) / wave * wave;
        for (int t = s + 1; t <= nlev && used < cap; t++)
            for (; head[t] < bucket[t].size() && used + boots(bucket[t][head[t]]) <= cap; head[t]++) {
                const int g = bucket[t][head[t]];
                placed.push_back(g);
                used += boots(g);
            }
        for (int g : placed) level[num_inputs + g] = s;
        for (int g : placed)
            for (int i = cons_off[g]; i < cons_off[g + 1]; i++)
                if (--waiting[cons[i]] == 0) make_ready(cons[i]);
    }
}

// Internal order (by level, bootstrapped gates before NOT/COPY in each level), descriptors and the
// output permutation of one level assignment, uploaded to the device (the current one).
// With nshards > 1 the schedule is shard `shard` of a netlist split across devices: every level keeps
// a contiguous run of its bootstrapped gates, cut so that the shards' bootstrap counts are balanced
// (a MUX counts two), and all of its NOT/COPY gates, which every shard evaluates itself.  The internal
// row order is the same for every shard, so a shard's outputs are rows out_row..out_row+gates-1 of
// each level in every shard's wire array.
cudaError_t build_schedule(int num_inputs, int num_gates, const int32_t *gates,
                           const int32_t *in_a, const int32_t *in_b, const int32_t *in_c, int nlev,
                           const std::vector<int> &level, Schedule &sc, int shard = 0, int nshards = 1) {
    std::vector<int> order(num_gates);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const int lx = level[num_inputs + x], ly = level[num_inputs + y];
        if (lx != ly) return lx < ly;
        return (gates[x] >= TFHEB_NOT) < (gates[y] >= TFHEB_NOT);
    });
    std::vector<int32_t> row_of(num_inputs + num_gates), perm(num_gates);
    for (int i = 0; i < num_inputs; i++) row_of[i] = i;
    for (int r = 0; r < num_gates; r++) {
        row_of[num_inputs + order[r]] = num_inputs + r;
        perm[r] = num_inputs + order[r];
    }
    std::vector<BootDescRows> bd;
    std::vector<GateDesc> gd;
    std::vector<UnaryDesc> ud;
    const int32_t mu8 = modswitch_to_torus32(1, 8), and_c = modswitch_to_torus32(-1, 8);
    int r = 0;
    for (int lv = 1; lv <= nlev; lv++) {
        // the level's rows [r0, r1): bootstrapped gates [r0, r0 + nb), then NOT/COPY
        const int r0 = r;
        int r1 = r0, nb = 0;
        int64_t total = 0;
        for (; r1 < num_gates && level[num_inputs + order[r1]] == lv; r1++)
            if (gates[order[r1]] < TFHEB_NOT) nb++, total += gates[order[r1]] == TFHEB_MUX ? 2 : 1;
        // this shard's gates [g0, g1) of the nb: gate i goes to shard (bootstraps before i) * nshards / total
        int g0 = nb, g1 = nb;
        {
            int64_t before = 0;
            for (int i = 0; i < nb; i++) {
                const int sh = total ? (int)std::min<int64_t>(nshards - 1, before * nshards / total) : 0;
                if (sh >= shard && g0 == nb) g0 = i;
                if (sh >= shard + 1) {
                    g1 = i;
                    break;
                }
                before += gates[order[r0 + i]] == TFHEB_MUX ? 2 : 1;
            }
        }
        Level L{(int)bd.size(), 0, (int)gd.size(), 0, (int)ud.size(), 0, num_inputs + r0 + g0};
        r = r1;
        for (int q = r0; q < r1; q++) {
            if (q - r0 < nb && (q - r0 < g0 || q - r0 >= g1)) continue;  // another shard's gate
            const int g = order[q], code = gates[g];
            const int xa = row_of[in_a[g]];
            if (code >= TFHEB_NOT) {
                ud.push_back(UnaryDesc{xa, num_inputs + q, code == TFHEB_NOT});
                continue;
            }
            const int xb = row_of[in_b[g]];
            const int local = (int)bd.size() - L.boot_off;
            if (code == TFHEB_MUX) {
                const int xc = row_of[in_c[g]];
                bd.push_back(BootDescRows{xa, xb, and_c, 1, 1, 0});
                bd.push_back(BootDescRows{xa, xc, and_c, -1, 1, 0});
                gd.push_back(GateDesc{local, local + 1, mu8});
            } else {
                int32_t cst, sa, sb;
                gate_form(code, &cst, &sa, &sb);
                bd.push_back(BootDescRows{xa, xb, cst, (int8_t)sa, (int8_t)sb, 0});
                gd.push_back(GateDesc{local, -1, 0});
            }
        }
        L.boots = (int)bd.size() - L.boot_off;
        L.gates = (int)gd.size() - L.gate_off;
        L.unaries = (int)ud.size() - L.unary_off;
        sc.max_boots = std::max(sc.max_boots, L.boots);
        sc.max_gates = std::max(sc.max_gates, L.gates);
        sc.levels.push_back(L);
    }
    auto alloc = [&](void **ptr, size_t bytes) { return bytes ? cudaMalloc(ptr, bytes) : cudaSuccess; };
    cudaError_t e = alloc((void **)&sc.d_boot, bd.size() * sizeof(BootDescRows));
    if (e == cudaSuccess) e = alloc((void **)&sc.d_gate, gd.size() * sizeof(GateDesc));
    if (e == cudaSuccess) e = alloc((void **)&sc.d_unary, ud.size() * sizeof(UnaryDesc));
    if (e == cudaSuccess) e = alloc((void **)&sc.d_out_perm, perm.size() * 4);
    if (e == cudaSuccess && !bd.empty())
        e = cudaMemcpy(sc.d_boot, bd.data(), bd.size() * sizeof(BootDescRows), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !gd.empty())
        e = cudaMemcpy(sc.d_gate, gd.data(), gd.size() * sizeof(GateDesc), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !ud.empty())
        e = cudaMemcpy(sc.d_unary, ud.data(), ud.size() * sizeof(UnaryDesc), cudaMemcpyHostToDevice);
    if (e == cudaSuccess && !perm.empty())
        e = cudaMemcpy(sc.d_out_perm, perm.data(), perm.size() * 4, cudaMemcpyHostToDevice);
    return e;
}

tfheb_status netlist_enqueue_run(tfheb_netlist *nl, CloudKey &ck, int32_t precision, int32_t *d_wires,
                                 int32_t use_graph, cudaStream_t s);

// Earliest level of every wire (inputs 0, a gate 1 + its deepest input) and the level count; an
// error message when a gate code is unknown or a gate reads a wire that is not earlier.
std::string earliest_levels(int num_inputs, int num_gates, const int32_t *gates, const int32_t *in_a,
                            const int32_t *in_b, const int32_t *in_c, std::vector<int> &level, int &nlev) {
    level.assign((size_t)num_inputs + num_gates, 0);
    for (int g = 0; g < num_gates; g++) {
        const int w = num_inputs + g, code = gates[g];
        if (code < 0 || code > TFHEB_COPY) return "netlist: unknown gate code at gate " + std::to_string(g);
        const int nin = code == TFHEB_MUX ? 3 : (code >= TFHEB_NOT ? 1 : 2);
        const int32_t *ins[3] = {in_a, in_b, in_c};
        int lv = 0;
        for (int k = 0; k < nin; k++) {
            if (!ins[k]) return "netlist: missing operand array";
            const int src = ins[k][g];
            if (src < 0 || src >= w) return "netlist: gate " + std::to_string(g) + " reads a later wire";
            lv = std::max(lv, level[src]);
        }
        level[w] = lv + 1;
    }
    nlev = num_gates ? *std::max_element(level.begin() + num_inputs, level.end()) : 0;
    return std::string();
}

}  // namespace

extern "C" {

tfheb_status tfheb_netlist_create(tfheb_cloud_key *c, int32_t num_inputs, int32_t num_gates, const int32_t *gates,
                                  const int32_t *in_a, const int32_t *in_b, const int32_t *in_c,
                                  tfheb_netlist **out) {
    if (!c || !out || num_inputs <= 0 || num_gates < 0 || (num_gates > 0 && (!gates || !in_a))) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    if (ck.device < 0) return nl_fail("cloud key is not on a device (call tfheb_cloud_key_to_device)");
    std::vector<int> level;
    int nlev = 0;
    const std::string bad = earliest_levels(num_inputs, num_gates, gates, in_a, in_b, in_c, level, nlev);
    if (!bad.empty()) return nl_fail(bad);
    auto *nl = new tfheb_netlist();
    nl->ck = c;
    nl->num_inputs = num_inputs;
    nl->num_gates = num_gates;
    cudaError_t e = cudaSetDevice(ck.device);
    for (int prec = 0; prec < 2 && e == cudaSuccess; prec++) {
        std::vector<int> lv(level);
        pack_levels(num_inputs, num_gates, gates, in_a, in_b, in_c, nlev, wave_bootstraps(ck, prec), lv);
        e = build_schedule(num_inputs, num_gates, gates, in_a, in_b, in_c, nlev, lv, nl->sched[prec]);
    }
    const tfheb_params &p = ck.p;
    const size_t rows = (size_t)num_inputs + num_gates;
    const int max_boots = std::max(nl->sched[0].max_boots, nl->sched[1].max_boots);
    const int max_gates = std::max(nl->sched[0].max_gates, nl->sched[1].max_gates);
    auto alloc = [&](void **ptr, size_t bytes) { return bytes ? cudaMalloc(ptr, bytes) : cudaSuccess; };
    if (e == cudaSuccess) e = alloc((void **)&nl->d_wires, rows * (p.n + 1) * 4);
    if (e == cudaSuccess) e = alloc((void **)&nl->d_bara, (size_t)max_boots * bara_stride_for(p) * 4);
    if (e == cudaSuccess) e = alloc((void **)&nl->d_acc, (size_t)max_boots * (p.k + 1) * p.N * 4);
    if (e == cudaSuccess) e = alloc((void **)&nl->d_ksin, (size_t)max_gates * (p.k * p.N + 1) * 4);
    if (e != cudaSuccess) {
        set_error(std::string("tfheb_netlist_create: ") + cudaGetErrorString(e));
        tfheb_netlist_free(nl);
        return e == cudaErrorMemoryAllocation ? TFHEB_ERR_NOMEM : TFHEB_ERR_CUDA;
    }
    *out = nl;
    return TFHEB_OK;
}

tfheb_status tfheb_netlist_info(const tfheb_netlist *nl, int32_t *num_levels, int32_t *max_width) {
    if (!nl) return TFHEB_ERR_INVALID;
    // both schedules have the same number of levels; the widths are those of the split-FP32 one
    const Schedule &sc = nl->sched[TFHEB_SPLIT_FP32];
    if (num_levels) *num_levels = (int32_t)sc.levels.size();
    if (max_width) {
        int w = 0;
        for (const auto &L : sc.levels) w = std::max(w, L.gates + L.unaries);
        *max_width = w;
    }
    return TFHEB_OK;
}

tfheb_status tfheb_netlist_run(tfheb_netlist *nl, int32_t precision, int32_t *d_wires, int32_t use_graph,
                               void *stream) {
    if (!nl || !d_wires) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(nl->ck->mu);
    CloudKey &ck = nl->ck->ck;
    tfheb_status st = prepare_device(ck, precision);
    if (st != TFHEB_OK) return st;
    if ((st = check_device_ptr(ck, d_wires, "tfheb_netlist_run: d_wires")) != TFHEB_OK) return st;
    cudaStream_t s = stream ? (cudaStream_t)stream : ck.stream;
    cudaError_t eo = nl->run_done ? cudaStreamWaitEvent(s, nl->run_done, 0)
                                  : cudaEventCreateWithFlags(&nl->run_done, cudaEventDisableTiming);
    if (eo != cudaSuccess) return nl_fail(std::string("tfheb_netlist_run: ") + cudaGetErrorString(eo), TFHEB_ERR_CUDA);
    st = netlist_enqueue_run(nl, ck, precision, d_wires, use_graph, s);
    eo = cudaEventRecord(nl->run_done, s);
    if (st == TFHEB_OK && eo != cudaSuccess)
        return nl_fail(std::string("tfheb_netlist_run: ") + cudaGetErrorString(eo), TFHEB_ERR_CUDA);
    return st;
}

}  // extern "C"

namespace {

// Evaluates the netlist on stream s: eagerly, or through the CUDA graph of (precision, d_wires),
// capturing it on the first graph run.
tfheb_status netlist_enqueue_run(tfheb_netlist *nl, CloudKey &ck, int32_t precision, int32_t *d_wires,
                                 int32_t use_graph, cudaStream_t s) {
    int kernels = 0;
    if (!use_graph) {
        const cudaError_t e = enqueue_netlist(nl, ck, precision, d_wires, s, &kernels);
        g_kernel_launches += kernels;
        if (e != cudaSuccess) return nl_fail(std::string("tfheb_netlist_run: ") + cudaGetErrorString(e), TFHEB_ERR_CUDA);
        return TFHEB_OK;
    }
    const auto key = std::make_pair((int)precision, (const int32_t *)d_wires);
    auto it = nl->graphs.find(key);
    if (it == nl->graphs.end()) {
        // blind-rotation launches set their shared-memory attribute outside the capture first
        cudaError_t e = enqueue_netlist(nl, ck, precision, d_wires, s, &kernels);
        g_kernel_launches += kernels;
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        cudaGraph_t g = nullptr;
        cudaGraphExec_t ge = nullptr;
        if (e == cudaSuccess) e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            const cudaError_t e1 = enqueue_netlist(nl, ck, precision, d_wires, s, &nl->sched[precision].graph_kernels);
            const cudaError_t e2 = cudaStreamEndCapture(s, &g);
            e = e1 != cudaSuccess ? e1 : e2;
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&ge, g, 0);
        if (e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            return nl_fail(std::string("tfheb_netlist_run (graph): ") + cudaGetErrorString(e), TFHEB_ERR_CUDA);
        }
        nl->graph_defs[key] = g;
        it = nl->graphs.emplace(key, ge).first;
        return TFHEB_OK;  // this call already evaluated the netlist eagerly
    }
    const cudaError_t e = cudaGraphLaunch(it->second, s);
    if (e != cudaSuccess) return nl_fail(std::string("tfheb_netlist_run: ") + cudaGetErrorString(e), TFHEB_ERR_CUDA);
    g_kernel_launches += nl->sched[precision].graph_kernels;
    return TFHEB_OK;
}

}  // namespace

extern "C" {

void tfheb_netlist_free(tfheb_netlist *nl) {
    if (!nl) return;
    cudaSetDevice(nl->ck->ck.device);
    for (auto &kv : nl->graphs) cudaGraphExecDestroy(kv.second);
    for (auto &kv : nl->graph_defs) cudaGraphDestroy(kv.second);
    if (nl->run_done) cudaEventDestroy(nl->run_done);
    for (auto &sc : nl->sched) sc.release();
    cudaFree(nl->d_wires);
    cudaFree(nl->d_bara);
    cudaFree(nl->d_acc);
    cudaFree(nl->d_ksin);
    delete nl;
}


// One batch of mixed gate types over rows of a device wire array: the launch sequence of one netlist
// level, with operand and output rows given by the caller.  Every operand is read before any output
// row is written, so outputs may overwrite operands of the same batch.
tfheb_status tfheb_gate_batch_mixed_device(tfheb_cloud_key *c, int32_t precision, int32_t count, const int32_t *gates,
                                           const int32_t *idx_a, const int32_t *idx_b, const int32_t *idx_c,
                                           const int32_t *out_idx, int32_t *d_wires, int32_t num_wires,
                                           void *stream) {
    if (!c || count < 0 || !d_wires || num_wires <= 0 || (count > 0 && (!gates || !idx_a || !out_idx)))
        return nl_fail("tfheb_gate_batch_mixed_device: invalid arguments");
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    tfheb_status st = prepare_device(ck, precision);
    if (st != TFHEB_OK) return st;
    if (count == 0) return TFHEB_OK;
    if ((st = check_device_ptr(ck, d_wires, "tfheb_gate_batch_mixed_device: d_wires")) != TFHEB_OK) return st;
    const tfheb_params &p = ck.p;
    const int n1 = p.n + 1, kN1 = p.k * p.N + 1, bs = bara_stride_for(p);
    auto row_ok = [&](const int32_t *idx, int g) { return idx && idx[g] >= 0 && idx[g] < num_wires; };
    // bootstrapped gates take scratch rows 0..nb-1 in batch order, NOT/COPY the rows after them
    std::vector<BootDescRows> bd;
    std::vector<GateDesc> gd;
    std::vector<UnaryDesc> ud;
    std::vector<int32_t> dst_boot, dst_unary;
    std::vector<char> written(num_wires, 0);
    const int32_t mu8 = modswitch_to_torus32(1, 8), and_c = modswitch_to_torus32(-1, 8);
    for (int g = 0; g < count; g++) {
        const int code = gates[g];
        const std::string at = " at gate " + std::to_string(g);
        if (code < 0 || code > TFHEB_COPY) return nl_fail("tfheb_gate_batch_mixed_device: unknown gate code" + at);
        if (!row_ok(out_idx, g)) return nl_fail("tfheb_gate_batch_mixed_device: output row out of range" + at);
        if (written[out_idx[g]]) return nl_fail("tfheb_gate_batch_mixed_device: output row written twice" + at);
        written[out_idx[g]] = 1;
        if (!row_ok(idx_a, g)) return nl_fail("tfheb_gate_batch_mixed_device: operand row out of range" + at);
        if (code >= TFHEB_NOT) {
            ud.push_back(UnaryDesc{idx_a[g], 0, code == TFHEB_NOT});
            dst_unary.push_back(out_idx[g]);
            continue;
        }
        if (!row_ok(idx_b, g) || (code == TFHEB_MUX && !row_ok(idx_c, g)))
            return nl_fail("tfheb_gate_batch_mixed_device: operand row out of range" + at);
        const int local = (int)bd.size();
        if (code == TFHEB_MUX) {
            bd.push_back(BootDescRows{idx_a[g], idx_b[g], and_c, 1, 1, 0});
            bd.push_back(BootDescRows{idx_a[g], idx_c[g], and_c, -1, 1, 0});
            gd.push_back(GateDesc{local, local + 1, mu8});
        } else {
            int32_t cst, sa, sb;
            gate_form(code, &cst, &sa, &sb);
            bd.push_back(BootDescRows{idx_a[g], idx_b[g], cst, (int8_t)sa, (int8_t)sb, 0});
            gd.push_back(GateDesc{local, -1, 0});
        }
        dst_boot.push_back(out_idx[g]);
    }
    const int nb = (int)gd.size(), nu = (int)ud.size(), boots = (int)bd.size();
    for (int u = 0; u < nu; u++) ud[u].dst = nb + u;
    std::vector<int32_t> perm(dst_boot);
    perm.insert(perm.end(), dst_unary.begin(), dst_unary.end());
    cudaStream_t s = stream ? (cudaStream_t)stream : ck.stream;
    // stream-ordered scratch: descriptors, rotation amounts, accumulators, extracted samples, results
    void *buf[8] = {nullptr};
    const size_t bytes[8] = {bd.size() * sizeof(BootDescRows), gd.size() * sizeof(GateDesc), ud.size() * sizeof(UnaryDesc),
                             perm.size() * 4, (size_t)boots * bs * 4, (size_t)boots * (p.k + 1) * p.N * 4,
                             (size_t)nb * kN1 * 4, (size_t)count * n1 * 4};
    cudaError_t e = cudaSuccess;
    for (int i = 0; i < 8 && e == cudaSuccess; i++)
        if (bytes[i]) e = cudaMallocAsync(&buf[i], bytes[i], s);
    const void *host[4] = {bd.data(), gd.data(), ud.data(), perm.data()};
    for (int i = 0; i < 4 && e == cudaSuccess; i++)
        if (bytes[i]) e = cudaMemcpyAsync(buf[i], host[i], bytes[i], cudaMemcpyHostToDevice, s);
    auto *d_tmp = static_cast<int32_t *>(buf[7]);
    int launches = 0;
    if (e == cudaSuccess && nb > 0) {
        const uint64_t interv = ((UINT64_C(1) << 63) / (uint64_t)(2 * p.N)) * 2;
        prologue_rows_kernel<<<boots, 256, 0, s>>>(static_cast<const BootDescRows *>(buf[0]),
                                                  reinterpret_cast<const uint32_t *>(d_wires), p.n, interv,
                                                  static_cast<int32_t *>(buf[4]), bs);
        e = cudaGetLastError();
        if (e == cudaSuccess)
            e = launch_blind_rotate(p, precision, ck.dbsk[precision], static_cast<int32_t *>(buf[4]), bs, boots, p.n,
                                    mu8, nullptr, static_cast<int32_t *>(buf[5]), s, ck.d_err, ck.stall_producer,
                                    ck.wait_timeout_ns, ck.br[precision]);
        if (e == cudaSuccess)
            e = launch_extract(p, static_cast<const GateDesc *>(buf[1]), nb, static_cast<int32_t *>(buf[5]),
                               static_cast<int32_t *>(buf[6]), kN1, s);
        if (e == cudaSuccess) e = launch_keyswitch(ck, nb, static_cast<int32_t *>(buf[6]), kN1, d_tmp, s);
        launches += 4;
    }
    if (e == cudaSuccess && nu > 0) {
        unary_rows_kernel<<<nu, 256, 0, s>>>(static_cast<const UnaryDesc *>(buf[2]),
                                             reinterpret_cast<const uint32_t *>(d_wires),
                                             reinterpret_cast<uint32_t *>(d_tmp), p.n);
        e = cudaGetLastError();
        launches += 1;
    }
    if (e == cudaSuccess) {
        permute_rows_kernel<<<count, 256, 0, s>>>(static_cast<const int32_t *>(buf[3]),
                                                  reinterpret_cast<const uint32_t *>(d_tmp),
                                                  reinterpret_cast<uint32_t *>(d_wires), p.n, 0);
        e = cudaGetLastError();
        launches += 1;
    }
    for (int i = 0; i < 8; i++)
        if (buf[i]) cudaFreeAsync(buf[i], s);
    g_kernel_launches += launches;
    if (e != cudaSuccess)
        return nl_fail(std::string("tfheb_gate_batch_mixed_device: ") + cudaGetErrorString(e), TFHEB_ERR_CUDA);
    return TFHEB_OK;
}


tfheb_status tfheb_netlist_multi_create(tfheb_cloud_key *const *cks, int32_t nkeys, int32_t num_inputs,
                                        int32_t num_gates, const int32_t *gates, const int32_t *in_a,
                                        const int32_t *in_b, const int32_t *in_c, tfheb_netlist_multi **out) {
    if (!cks || nkeys < 1 || !out || num_inputs <= 0 || num_gates < 0 || (num_gates > 0 && (!gates || !in_a)))
        return nl_fail("tfheb_netlist_multi_create: invalid arguments");
    for (int k = 0; k < nkeys; k++) {
        if (!cks[k]) return nl_fail("tfheb_netlist_multi_create: key " + std::to_string(k) + " is NULL");
        for (int j = 0; j < k; j++)
            if (cks[j] == cks[k]) return nl_fail("tfheb_netlist_multi_create: key " + std::to_string(k) + " repeats key " + std::to_string(j));
        const tfheb_params &p0 = cks[0]->ck.p, &pk = cks[k]->ck.p;
        if (pk.n != p0.n || pk.N != p0.N || pk.k != p0.k || pk.l != p0.l || pk.Bgbit != p0.Bgbit ||
            pk.ks_t != p0.ks_t || pk.ks_basebit != p0.ks_basebit)
            return nl_fail("tfheb_netlist_multi_create: key " + std::to_string(k) + " has another parameter set than key 0");
    }
    for (int k = 0; k < nkeys; k++)
        if (cks[k]->ck.device < 0)
            return nl_fail("tfheb_netlist_multi_create: key " + std::to_string(k) + " is not on a device");
    std::vector<int> level;
    int nlev = 0;
    const std::string bad = earliest_levels(num_inputs, num_gates, gates, in_a, in_b, in_c, level, nlev);
    if (!bad.empty()) return nl_fail(bad);
    auto *nl = new tfheb_netlist_multi();
    nl->cks.assign(cks, cks + nkeys);
    nl->num_inputs = num_inputs;
    nl->num_gates = num_gates;
    nl->nlev = nlev;
    nl->shards.resize(nkeys);
    const tfheb_params &p = cks[0]->ck.p;
    const size_t rows = (size_t)num_inputs + num_gates;
    cudaError_t e = cudaSuccess;
    for (int prec = 0; prec < 2 && e == cudaSuccess; prec++) {
        // the levels are packed for the waves of all keys together
        int wave = 0;
        for (int k = 0; k < nkeys; k++) wave += wave_bootstraps(cks[k]->ck, prec);
        std::vector<int> lv(level);
        pack_levels(num_inputs, num_gates, gates, in_a, in_b, in_c, nlev, wave, lv);
        for (int k = 0; k < nkeys && e == cudaSuccess; k++) {
            e = cudaSetDevice(cks[k]->ck.device);
            if (e == cudaSuccess)
                e = build_schedule(num_inputs, num_gates, gates, in_a, in_b, in_c, nlev, lv, nl->shards[k].sched[prec],
                                   k, nkeys);
        }
    }
    auto alloc = [&](void **ptr, size_t bytes) { return bytes ? cudaMalloc(ptr, bytes) : cudaSuccess; };
    for (int k = 0; k < nkeys && e == cudaSuccess; k++) {
        auto &sh = nl->shards[k];
        const int dev = cks[k]->ck.device;
        e = cudaSetDevice(dev);
        for (int j = 0; j < nkeys && e == cudaSuccess; j++) {  // peer access for the all-gather copies
            const int other = cks[j]->ck.device;
            int can = 0;
            if (other == dev || cudaDeviceCanAccessPeer(&can, dev, other) != cudaSuccess || !can) continue;
            if (cudaDeviceEnablePeerAccess(other, 0) != cudaSuccess) cudaGetLastError();  // already enabled
        }
        const int max_boots = std::max(sh.sched[0].max_boots, sh.sched[1].max_boots);
        const int max_gates = std::max(sh.sched[0].max_gates, sh.sched[1].max_gates);
        if (e == cudaSuccess) e = alloc((void **)&sh.d_wires, rows * (p.n + 1) * 4);
        if (e == cudaSuccess) e = alloc((void **)&sh.d_bara, (size_t)max_boots * bara_stride_for(p) * 4);
        if (e == cudaSuccess) e = alloc((void **)&sh.d_acc, (size_t)max_boots * (p.k + 1) * p.N * 4);
        if (e == cudaSuccess) e = alloc((void **)&sh.d_ksin, (size_t)max_gates * (p.k * p.N + 1) * 4);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sh.copied, cudaEventDisableTiming);
        if (e == cudaSuccess && k == 0) e = alloc((void **)&nl->d_user, rows * (p.n + 1) * 4);
    }
    if (e != cudaSuccess) {
        set_error(std::string("tfheb_netlist_multi_create: ") + cudaGetErrorString(e));
        tfheb_netlist_multi_free(nl);
        return e == cudaErrorMemoryAllocation ? TFHEB_ERR_NOMEM : TFHEB_ERR_CUDA;
    }
    *out = nl;
    return TFHEB_OK;
}

tfheb_status tfheb_netlist_multi_run(tfheb_netlist_multi *nl, int32_t precision, int32_t *wires) {
    if (!nl || !wires || (precision != TFHEB_FP64 && precision != TFHEB_SPLIT_FP32))
        return nl_fail("tfheb_netlist_multi_run: invalid arguments");
    const int K = (int)nl->cks.size();
    // lock the keys in address order, so that runs over overlapping key sets cannot deadlock
    std::vector<tfheb_cloud_key *> order(nl->cks);
    std::sort(order.begin(), order.end());
    std::vector<std::unique_lock<std::mutex>> locks;
    for (auto *c : order) locks.emplace_back(c->mu);
    for (int k = 0; k < K; k++) {
        const tfheb_status st = prepare_device(nl->cks[k]->ck, precision);
        if (st != TFHEB_OK) return st;
    }
    const tfheb_params &p = nl->cks[0]->ck.p;
    const size_t n1 = (size_t)p.n + 1;
    auto dev = [&](int k) { return nl->cks[k]->ck.device; };
    auto strm = [&](int k) { return nl->cks[k]->ck.stream; };
    cudaError_t e = cudaSuccess;
    int launches = 0;
    for (int k = 0; k < K && e == cudaSuccess; k++) {
        e = cudaSetDevice(dev(k));
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(nl->shards[k].d_wires, wires, (size_t)nl->num_inputs * n1 * 4, cudaMemcpyHostToDevice,
                                strm(k));
    }
    for (int lv = 0; lv < nl->nlev && e == cudaSuccess; lv++) {
        // each key: wait for the other keys' outputs of the previous level, then run its shard
        for (int k = 0; k < K && e == cudaSuccess; k++) {
            auto &sh = nl->shards[k];
            e = cudaSetDevice(dev(k));
            for (int j = 0; j < K && e == cudaSuccess && lv > 0; j++)
                if (j != k) e = cudaStreamWaitEvent(strm(k), nl->shards[j].copied, 0);
            if (e == cudaSuccess)
                e = enqueue_level(sh.sched[precision], sh.sched[precision].levels[lv], nl->cks[k]->ck, precision,
                                  LevelScratch{sh.d_wires, sh.d_bara, sh.d_acc, sh.d_ksin}, strm(k), launches);
        }
        // all-gather: each key copies its shard's output rows into every other key's wire array
        for (int k = 0; k < K && e == cudaSuccess; k++) {
            auto &sh = nl->shards[k];
            const Level &L = sh.sched[precision].levels[lv];
            e = cudaSetDevice(dev(k));
            for (int j = 0; j < K && e == cudaSuccess && L.gates > 0; j++)
                if (j != k)
                    e = cudaMemcpyPeerAsync(nl->shards[j].d_wires + (size_t)L.out_row * n1, dev(j),
                                            sh.d_wires + (size_t)L.out_row * n1, dev(k), (size_t)L.gates * n1 * 4,
                                            strm(k));
            if (e == cudaSuccess) e = cudaEventRecord(sh.copied, strm(k));
        }
    }
    // key 0 holds every wire once the last level's copies into it are done
    if (e == cudaSuccess) e = cudaSetDevice(dev(0));
    for (int j = 1; j < K && e == cudaSuccess && nl->nlev > 0; j++) e = cudaStreamWaitEvent(strm(0), nl->shards[j].copied, 0);
    if (e == cudaSuccess && nl->num_gates > 0) {
        const Schedule &sc = nl->shards[0].sched[precision];
        permute_rows_kernel<<<nl->num_gates, 256, 0, strm(0)>>>(sc.d_out_perm,
                                                               reinterpret_cast<const uint32_t *>(nl->shards[0].d_wires),
                                                               reinterpret_cast<uint32_t *>(nl->d_user), p.n,
                                                               nl->num_inputs);
        e = cudaGetLastError();
        launches += 1;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(wires + (size_t)nl->num_inputs * n1, nl->d_user + (size_t)nl->num_inputs * n1,
                                (size_t)nl->num_gates * n1 * 4, cudaMemcpyDeviceToHost, strm(0));
    }
    g_kernel_launches += launches;
    // drain every stream, also after an error, before reporting
    for (int k = 0; k < K; k++) {
        cudaSetDevice(dev(k));
        const cudaError_t es = cudaStreamSynchronize(strm(k));
        if (e == cudaSuccess) e = es;
    }
    if (e != cudaSuccess) return nl_fail(std::string("tfheb_netlist_multi_run: ") + cudaGetErrorString(e), TFHEB_ERR_CUDA);
    for (int k = 0; k < K; k++) {
        cudaSetDevice(dev(k));
        const tfheb_status st = check_device_error(nl->cks[k]->ck);
        if (st != TFHEB_OK) return st;
    }
    return TFHEB_OK;
}

void tfheb_netlist_multi_free(tfheb_netlist_multi *nl) {
    if (!nl) return;
    for (size_t k = 0; k < nl->shards.size(); k++) {
        auto &sh = nl->shards[k];
        cudaSetDevice(nl->cks[k]->ck.device);
        for (auto &sc : sh.sched) sc.release();
        cudaFree(sh.d_wires);
        cudaFree(sh.d_bara);
        cudaFree(sh.d_acc);
        cudaFree(sh.d_ksin);
        if (sh.copied) cudaEventDestroy(sh.copied);
        if (k == 0) cudaFree(nl->d_user);
    }
    delete nl;
}

}  // extern "C"
