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
#include <cuda_runtime.h>

#include <algorithm>
#include <map>
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

// bootstrap-free gates: NOT negates, COPY copies (boot-gates.cpp:164-178)
__global__ void unary_rows_kernel(const UnaryDesc *__restrict__ desc, uint32_t *__restrict__ wires, int n) {
    const UnaryDesc d = desc[blockIdx.x];
    const uint32_t *src = wires + (size_t)d.src * (n + 1);
    uint32_t *dst = wires + (size_t)d.dst * (n + 1);
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
    int out_row;             // first internal row of the level's outputs
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
};

using namespace tfheb;

namespace {

tfheb_status nl_fail(const std::string &msg, tfheb_status st = TFHEB_ERR_INVALID) {
    set_error(msg);
    return st;
}

// Enqueues the whole level sequence on stream s (also used inside stream capture).
cudaError_t enqueue_netlist(tfheb_netlist *nl, CloudKey &ck, int precision, int32_t *user_wires, cudaStream_t s,
                            int *kernels) {
    const tfheb_params &p = ck.p;
    const int n1 = p.n + 1, kN1 = p.k * p.N + 1, bs = bara_stride_for(p);
    const uint64_t interv = ((UINT64_C(1) << 63) / (uint64_t)(2 * p.N)) * 2;
    cudaError_t e = cudaMemcpyAsync(nl->d_wires, user_wires, (size_t)nl->num_inputs * n1 * 4,
                                    cudaMemcpyDeviceToDevice, s);
    int launches = 0;
    const Schedule &sc = nl->sched[precision];
    for (const Level &L : sc.levels) {
        if (e != cudaSuccess) break;
        if (L.boots > 0) {
            prologue_rows_kernel<<<L.boots, 256, 0, s>>>(sc.d_boot + L.boot_off,
                                                         reinterpret_cast<const uint32_t *>(nl->d_wires), p.n, interv,
                                                         nl->d_bara, bs);
            if ((e = cudaGetLastError()) != cudaSuccess) break;
            e = launch_blind_rotate(p, precision, ck.dbsk[precision], nl->d_bara, bs, L.boots, p.n,
                                    modswitch_to_torus32(1, 8), nullptr, nl->d_acc, s, ck.d_err, ck.stall_producer,
                                    ck.wait_timeout_ns, ck.br_variant[precision]);
            if (e != cudaSuccess) break;
            e = launch_extract(p, sc.d_gate + L.gate_off, L.gates, nl->d_acc, nl->d_ksin, kN1, s);
            if (e != cudaSuccess) break;
            e = launch_keyswitch(ck, L.gates, nl->d_ksin, kN1,
                                 nl->d_wires + (size_t)L.out_row * n1, s);
            launches += 4;
        }
        if (e == cudaSuccess && L.unaries > 0) {
            unary_rows_kernel<<<L.unaries, 256, 0, s>>>(sc.d_unary + L.unary_off,
                                                         reinterpret_cast<uint32_t *>(nl->d_wires), p.n);
            e = cudaGetLastError();
            launches += 1;
        }
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
    const int v = ck.br_variant[precision];
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
// output permutation of one level assignment, uploaded to the device.
cudaError_t build_schedule(int num_inputs, int num_gates, const int32_t *gates,
                           const int32_t *in_a, const int32_t *in_b, const int32_t *in_c, int nlev,
                           const std::vector<int> &level, Schedule &sc) {
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
        Level L{(int)bd.size(), 0, (int)gd.size(), 0, (int)ud.size(), 0, num_inputs + r};
        for (; r < num_gates && level[num_inputs + order[r]] == lv; r++) {
            const int g = order[r], code = gates[g];
            const int xa = row_of[in_a[g]];
            if (code >= TFHEB_NOT) {
                ud.push_back(UnaryDesc{xa, num_inputs + r, code == TFHEB_NOT});
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

}  // namespace

extern "C" {

tfheb_status tfheb_netlist_create(tfheb_cloud_key *c, int32_t num_inputs, int32_t num_gates, const int32_t *gates,
                                  const int32_t *in_a, const int32_t *in_b, const int32_t *in_c,
                                  tfheb_netlist **out) {
    if (!c || !out || num_inputs <= 0 || num_gates < 0 || (num_gates > 0 && (!gates || !in_a))) return TFHEB_ERR_INVALID;
    std::lock_guard<std::mutex> lock(c->mu);
    CloudKey &ck = c->ck;
    if (ck.device < 0) return nl_fail("cloud key is not on a device (call tfheb_cloud_key_to_device)");
    // levels
    std::vector<int> level(num_inputs + num_gates, 0);
    for (int g = 0; g < num_gates; g++) {
        const int w = num_inputs + g, code = gates[g];
        if (code < 0 || code > TFHEB_COPY) return nl_fail("netlist: unknown gate code at gate " + std::to_string(g));
        const int nin = code == TFHEB_MUX ? 3 : (code >= TFHEB_NOT ? 1 : 2);
        const int32_t *ins[3] = {in_a, in_b, in_c};
        int lv = 0;
        for (int k = 0; k < nin; k++) {
            if (!ins[k]) return nl_fail("netlist: missing operand array");
            const int src = ins[k][g];
            if (src < 0 || src >= w) return nl_fail("netlist: gate " + std::to_string(g) + " reads a later wire");
            lv = std::max(lv, level[src]);
        }
        level[w] = lv + 1;
    }
    const int nlev = num_gates ? *std::max_element(level.begin() + num_inputs, level.end()) : 0;
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
    cudaStream_t s = stream ? (cudaStream_t)stream : ck.stream;
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

void tfheb_netlist_free(tfheb_netlist *nl) {
    if (!nl) return;
    cudaSetDevice(nl->ck->ck.device);
    for (auto &kv : nl->graphs) cudaGraphExecDestroy(kv.second);
    for (auto &kv : nl->graph_defs) cudaGraphDestroy(kv.second);
    for (auto &sc : nl->sched) sc.release();
    cudaFree(nl->d_wires);
    cudaFree(nl->d_bara);
    cudaFree(nl->d_acc);
    cudaFree(nl->d_ksin);
    delete nl;
}

}  // extern "C"
