// Planned refit: the bottom-up box pass of BVHRT-Core/src/LBVH.cu:465-570 on
// a resident topology, organised so that every node's box is computed in
// shared memory by the CTA that owns its subtree.
//
// A refit plan cuts the tree into units: subtrees of at most kUnitInputs
// inputs whose parent holds more.  At level 0 the inputs are the triangles
// (leaves); at level k > 0 the inputs are the roots of the level k-1 units
// and the units cover the nodes above them.  Units are packed into CTAs of
// at most kCtaInputs inputs, each CTA getting its units' inputs and internal
// nodes as contiguous slot ranges with CTA-local links (parent slot, child
// slots).  The last level has one unit, rooted at the tree's root.
//
// A refit is one launch per level (two or three for millions of triangles):
// a CTA loads its inputs' boxes (level 0: the triangles' three vertices;
// later levels: the boxes the level below wrote), then climbs from every
// input with shared-memory arrival counters -- the second arrival at a node
// unites its children's boxes -- and writes every box and area it computes
// to the tree.  Plan arrays are read in slot order (coalesced); the climb
// itself never leaves the SM.  The boxes equal those of the arrival-counter
// climb over global memory (the same unions of the same boxes; min/max are
// exact) and the areas are computed from them in the same order.
//
// A plan depends only on the topology.  It is built on the second refit after
// a build or an optimiser changed the topology (that call synchronises the
// context's stream while it builds the plan; the first refit climbs over
// global memory, so a topology refit only once never pays for a plan) and
// reused by every later refit of the same tree.

#include <vector>

#include "common.cuh"
#include "internal.h"

namespace atr {

int exclusive_scan_u32(atr_ctx* ctx, const uint32_t* in, uint32_t* out, uint64_t n, uint32_t* d_total);

namespace {

constexpr int kUnitInputs = 256;    // inputs per unit, at most
constexpr int kCtaInputs = 512;     // inputs per CTA, at most (units start in [c, c+1) * kUnitInputs)
constexpr int kRefitThreads = 256;  // two inputs per thread
constexpr uint16_t kNoSlot = 0xffffu;
// Dynamic shared memory of a refit CTA: min and max boxes of every input and
// internal slot (3 floats each); per internal slot its arrival counter, node,
// child links and parent slot.
constexpr size_t kRefitSmem = (size_t)2 * kCtaInputs * 3 * 4 * 2 + (size_t)kCtaInputs * (4 + 4 + 4 + 2);
constexpr uint16_t kInputBit = 0x8000u;  // child link to an input slot (else an internal slot)

static_assert(kCtaInputs == 2 * kUnitInputs, "CTA capacity: one unit range plus one unit");
static_assert(kCtaInputs <= (int)kInputBit, "local slots fit in 15 bits");

// ---- plan construction ---------------------------------------------------------

// Inputs of level k climb towards the root passing their input counts
// through exchange slots (zero = empty; counts are never zero): the first
// arrival at a node leaves its count and stops, the second adds the two and
// goes on.  cnt[v] = inputs below v for every node at or above the inputs.
__global__ void __launch_bounds__(256) k_plan_count(const int32_t* __restrict__ parent, const int32_t* __restrict__ inputs,
                                                    uint32_t n_inputs, int32_t* __restrict__ cnt,
                                                    int32_t* __restrict__ xslot) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_inputs) return;
    int v = inputs[i];
    int c = 1;
    cnt[v] = 1;
    int p = parent[v];
    while (p >= 0) {
        const int other = atomicExch(&xslot[p], c);
        if (other == 0) return;
        c += other;
        cnt[p] = c;
        p = parent[p];
    }
}

// Level-0 inputs are the leaves [n-1, 2n-2].
__global__ void __launch_bounds__(256) k_plan_leaves(uint32_t n, int32_t* __restrict__ inputs) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) inputs[i] = (int32_t)(n - 1 + i);
}

// Unit roots of the level: nodes at or above the inputs holding at most
// kUnitInputs inputs whose parent holds more (or the tree's root).
// flag[v] = 1 for a unit root, size[v] = its input count (0 elsewhere).
__global__ void __launch_bounds__(256) k_plan_roots(uint32_t nodes, const int32_t* __restrict__ parent,
                                                    const int32_t* __restrict__ cnt, uint32_t* __restrict__ flag,
                                                    uint32_t* __restrict__ size) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nodes) return;
    const int c = cnt[v];
    const int p = parent[v];
    const bool root = c >= 1 && c <= kUnitInputs && (p < 0 || cnt[p] > kUnitInputs);
    flag[v] = root ? 1u : 0u;
    size[v] = root ? (uint32_t)c : 0u;
}

// Unit list in node order: unit u = uidx[v] for the unit root v, its inputs
// start at ustart[u] (exclusive scan of the sizes), internal slots at
// ustart[u] - u.
__global__ void __launch_bounds__(256) k_plan_units(uint32_t nodes, const uint32_t* __restrict__ flag,
                                                    const uint32_t* __restrict__ uidx,
                                                    const uint32_t* __restrict__ sstart,
                                                    uint32_t* __restrict__ ustart, int32_t* __restrict__ unit_of,
                                                    int32_t* __restrict__ next_inputs) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nodes || !flag[v]) return;
    const uint32_t u = uidx[v];
    ustart[u] = sstart[v];
    unit_of[v] = (int32_t)u;
    next_inputs[u] = (int32_t)v;  // the inputs of the next level
}

// First unit of every CTA: CTA c takes the units whose first input slot lies
// in [c, c+1) * kUnitInputs.  cta_first[c] = the first such unit (U when
// none), written by the unit that crosses into c.
__global__ void __launch_bounds__(256) k_plan_ctas(uint32_t U, uint32_t ctas, const uint32_t* __restrict__ ustart,
                                                   uint32_t* __restrict__ cta_first) {
    const uint32_t u = blockIdx.x * blockDim.x + threadIdx.x;
    if (u > U) return;
    const uint32_t c_hi = u < U ? ustart[u] / kUnitInputs : ctas;  // CTAs whose first unit is u: (c_lo, c_hi]
    const uint32_t c_lo = u == 0 ? 0u : ustart[u - 1] / kUnitInputs + 1;
    for (uint32_t c = c_lo; c <= c_hi && c <= ctas; ++c) cta_first[c] = u;
}

// Every node inside a unit (at or above the inputs, at most kUnitInputs
// inputs) climbs to its unit root: key 2u for an input of unit u, 2u + 1 for
// an internal node.  rel[v] = 1 for these nodes (0 elsewhere).
__global__ void __launch_bounds__(256) k_plan_keys(uint32_t nodes, const int32_t* __restrict__ parent,
                                                   const int32_t* __restrict__ cnt, const uint32_t* __restrict__ flag,
                                                   const uint8_t* __restrict__ is_input,
                                                   const int32_t* __restrict__ unit_of, uint32_t* __restrict__ key,
                                                   uint32_t* __restrict__ rel) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nodes) return;
    const int c = cnt[v];
    const bool in_unit = c >= 1 && c <= kUnitInputs;  // else below the inputs, or above every unit
    rel[v] = in_unit ? 1u : 0u;
    if (!in_unit) return;
    int r = (int)v;
    while (!flag[r]) r = parent[r];
    key[v] = 2u * (uint32_t)unit_of[r] + (is_input[v] ? 0u : 1u);
}

// The unit's nodes in node order, compacted for the sort.
__global__ void __launch_bounds__(256) k_plan_compact(uint32_t nodes, const uint32_t* __restrict__ rel,
                                                      const uint32_t* __restrict__ pos, const uint32_t* __restrict__ key,
                                                      uint32_t* __restrict__ ckey, uint32_t* __restrict__ cnode) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nodes || !rel[v]) return;
    ckey[pos[v]] = key[v];
    cnode[pos[v]] = v;
}

// After a stable sort by key, unit u's inputs and then its internal nodes sit
// in node order from position 2 * ustart[u] - u: each node's slot follows
// from its position.
__global__ void __launch_bounds__(256) k_plan_slots(uint32_t count, const uint32_t* __restrict__ skey,
                                                    const uint32_t* __restrict__ snode,
                                                    const uint32_t* __restrict__ ustart, uint32_t U, uint32_t total,
                                                    int32_t* __restrict__ gslot, int32_t* __restrict__ gunit) {
    const uint32_t q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= count) return;
    const uint32_t k = skey[q], u = k >> 1, v = snode[q];
    const uint32_t size = (u + 1 < U ? ustart[u + 1] : total) - ustart[u];
    const uint32_t g = 2 * ustart[u] - u;  // first position of the unit
    gunit[v] = (int32_t)u;
    gslot[v] = (k & 1u) ? (int32_t)(ustart[u] - u + (q - g - size)) : (int32_t)(ustart[u] + (q - g));
}

struct LevelOut {
    uint32_t *cta_first, *cta_in, *cta_int;
    int32_t *in_src, *in_node, *it_node;
    uint16_t *in_par, *it_par;
    uint32_t* it_kids;
};

// CTA-local slot offsets of every CTA: inputs from its first unit's start,
// internal slots from that start minus the unit index.
__global__ void __launch_bounds__(256) k_plan_cta_offsets(uint32_t U, uint32_t ctas, uint32_t total_inputs,
                                                          const uint32_t* __restrict__ ustart, LevelOut o) {
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c > ctas) return;
    const uint32_t u = o.cta_first[c];
    const uint32_t in0 = u < U ? ustart[u] : total_inputs;
    o.cta_in[c] = in0;
    o.cta_int[c] = in0 - u;
}

// Plan entries of every node inside a unit, with links as CTA-local slots.
__global__ void __launch_bounds__(256) k_plan_fill(uint32_t nodes, int level, const int32_t* __restrict__ parent,
                                                   const int32_t* __restrict__ left, const int32_t* __restrict__ right,
                                                   const int32_t* __restrict__ data, const int32_t* __restrict__ cnt,
                                                   const uint32_t* __restrict__ flag,
                                                   const uint8_t* __restrict__ is_input,
                                                   const int32_t* __restrict__ gslot, const int32_t* __restrict__ gunit,
                                                   const uint32_t* __restrict__ ustart, LevelOut o) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nodes) return;
    const int c = cnt[v];
    if (c < 1 || c > kUnitInputs) return;
    const uint32_t u = (uint32_t)gunit[v];
    const uint32_t cta = ustart[u] / kUnitInputs;
    const uint32_t in0 = o.cta_in[cta], int0 = o.cta_int[cta];
    const uint16_t par = flag[v] ? kNoSlot : (uint16_t)(gslot[parent[v]] - (int32_t)int0);
    const int32_t s = gslot[v];
    if (is_input[v]) {
        o.in_src[s] = level == 0 ? data[v] : (int32_t)v;
        o.in_node[s] = (int32_t)v;
        o.in_par[s] = par;
    } else {
        auto link = [&](int ch) -> uint32_t {
            return is_input[ch] ? ((uint32_t)(gslot[ch] - (int32_t)in0) | kInputBit) : (uint32_t)(gslot[ch] - (int32_t)int0);
        };
        o.it_node[s] = (int32_t)v;
        o.it_par[s] = par;
        o.it_kids[s] = link(left[v]) | (link(right[v]) << 16);
    }
}

__global__ void __launch_bounds__(256) k_mark_inputs(const int32_t* __restrict__ inputs, uint32_t count,
                                                     uint8_t* __restrict__ is_input) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) is_input[inputs[i]] = 1;
}

// ---- the refit -----------------------------------------------------------------

// One CTA of one level: inputs' boxes into shared memory, a climb from every
// input with shared arrival counters that touches shared memory only, then
// every box the CTA computed (and at level 0 the leaves' boxes) with its area
// into the tree.  Shared boxes: inputs at [0, kCtaInputs), internal slots at
// kCtaInputs + j.
__global__ void __launch_bounds__(kRefitThreads) k_refit_level(int level, const uint32_t* __restrict__ cta_in,
                                                               const uint32_t* __restrict__ cta_int,
                                                               const int32_t* __restrict__ in_src,
                                                               const int32_t* __restrict__ in_node,
                                                               const uint16_t* __restrict__ in_par,
                                                               const int32_t* __restrict__ it_node,
                                                               const uint16_t* __restrict__ it_par,
                                                               const uint32_t* __restrict__ it_kids,
                                                               const float4* __restrict__ verts,
                                                               float4* __restrict__ bmin, float4* __restrict__ bmax,
                                                               float* __restrict__ area) {
    extern __shared__ __align__(16) float s_refit[];
    float (*s_mn)[3] = reinterpret_cast<float (*)[3]>(s_refit);
    float (*s_mx)[3] = reinterpret_cast<float (*)[3]>(s_refit + 6 * kCtaInputs);
    int* s_arrive = reinterpret_cast<int*>(s_refit + 12 * kCtaInputs);
    int* s_node = s_arrive + kCtaInputs;
    uint32_t* s_kids = reinterpret_cast<uint32_t*>(s_node + kCtaInputs);
    uint16_t* s_par = reinterpret_cast<uint16_t*>(s_kids + kCtaInputs);
    const uint32_t i0 = cta_in[blockIdx.x], i1 = cta_in[blockIdx.x + 1];
    const uint32_t j0 = cta_int[blockIdx.x], j1 = cta_int[blockIdx.x + 1];
    const int nin = (int)(i1 - i0), nint = (int)(j1 - j0);
    // The internal slots' links come in once, coalesced; the climb then
    // touches shared memory only (and stores the boxes it computes).
    for (int j = threadIdx.x; j < nint; j += kRefitThreads) {
        s_arrive[j] = 0;
        s_node[j] = it_node[j0 + j];
        s_kids[j] = it_kids[j0 + j];
        s_par[j] = it_par[j0 + j];
    }
    for (int i = threadIdx.x; i < nin; i += kRefitThreads) {
        float mn[3], mx[3];
        if (level == 0) {
            const uint32_t tri = (uint32_t)in_src[i0 + i];
            const float4 a = __ldg(verts + 3 * (size_t)tri), b = __ldg(verts + 3 * (size_t)tri + 1),
                         c = __ldg(verts + 3 * (size_t)tri + 2);
            mn[0] = fminf(fminf(a.x, b.x), c.x); mn[1] = fminf(fminf(a.y, b.y), c.y); mn[2] = fminf(fminf(a.z, b.z), c.z);
            mx[0] = fmaxf(fmaxf(a.x, b.x), c.x); mx[1] = fmaxf(fmaxf(a.y, b.y), c.y); mx[2] = fmaxf(fmaxf(a.z, b.z), c.z);
        } else {
            const int node = in_src[i0 + i];
            const float4 a = bmin[node], b = bmax[node];
            mn[0] = a.x; mn[1] = a.y; mn[2] = a.z;
            mx[0] = b.x; mx[1] = b.y; mx[2] = b.z;
        }
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            s_mn[i][k] = mn[k];
            s_mx[i][k] = mx[k];
        }
    }
    __syncthreads();
    for (int i = threadIdx.x; i < nin; i += kRefitThreads) {
        uint16_t p = in_par[i0 + i];
        while (p != kNoSlot) {
            __threadfence_block();
            if (atomicAdd(&s_arrive[p], 1) == 0) break;  // first of the two children
            __threadfence_block();
            const uint32_t kids = s_kids[p];
            const int lc = (kids & kInputBit) ? (int)(kids & 0x7fffu) : kCtaInputs + (int)(kids & 0x7fffu);
            const uint32_t hi = kids >> 16;
            const int rc = (hi & kInputBit) ? (int)(hi & 0x7fffu) : kCtaInputs + (int)(hi & 0x7fffu);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                s_mn[kCtaInputs + p][k] = fminf(s_mn[lc][k], s_mn[rc][k]);
                s_mx[kCtaInputs + p][k] = fmaxf(s_mx[lc][k], s_mx[rc][k]);
            }
            p = s_par[p];
        }
    }
    __syncthreads();
    // Every box the CTA computed goes to the tree with its area (the leaves'
    // at level 0; later levels' inputs are boxes already written).
    auto put = [&](int slot, int node) {
        const float4 a = make_float4(s_mn[slot][0], s_mn[slot][1], s_mn[slot][2], 0.0f);
        const float4 b = make_float4(s_mx[slot][0], s_mx[slot][1], s_mx[slot][2], 0.0f);
        bmin[node] = a;
        bmax[node] = b;
        area[node] = box_area(a, b);
    };
    if (level == 0)
        for (int i = threadIdx.x; i < nin; i += kRefitThreads) put(i, in_node[i0 + i]);
    for (int j = threadIdx.x; j < nint; j += kRefitThreads) put(kCtaInputs + j, s_node[j]);
}

}  // namespace

void tree_topology_changed(atr_tree* t) {
    refit_plan_free(t->ctx, t->refit_plan);
    t->refit_plan = nullptr;
    t->no_refit_plan = false;
    t->refits = 0;
}

void refit_plan_free(atr_ctx* ctx, RefitPlan* p) {
    if (!p) return;
    for (void* b : p->blocks) ctx->release(b);
    delete p;
}

// Builds the plan of the topology (parent/left/right/data of n triangles).
int refit_plan_build(atr_ctx* ctx, uint32_t n, const TreeOut& t, RefitPlan** out) {
    *out = nullptr;
    cudaStream_t s = ctx->stream;
    const uint32_t nodes = 2 * n - 1;
    ATR_CUDA(cudaFuncSetAttribute(k_refit_level, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kRefitSmem));
    // Node-indexed scratch of the construction, and the sort's pairs.
    void* scratch = nullptr;
    const size_t nb4 = align256((size_t)nodes * 4);
    ATR_TRY(ctx->alloc(&scratch, 12 * nb4 + align256(nodes)));
    char* q = static_cast<char*>(scratch);
    auto take = [&](size_t b) { char* r = q; q += b; return r; };
    int32_t* cnt = reinterpret_cast<int32_t*>(take(nb4));
    int32_t* xslot = reinterpret_cast<int32_t*>(take(nb4));
    uint32_t* flag = reinterpret_cast<uint32_t*>(take(nb4));
    uint32_t* size = reinterpret_cast<uint32_t*>(take(nb4));
    uint32_t* uidx = reinterpret_cast<uint32_t*>(take(nb4));
    uint32_t* sstart = reinterpret_cast<uint32_t*>(take(nb4));
    int32_t* unit_of = reinterpret_cast<int32_t*>(take(nb4));
    int32_t* gslot = reinterpret_cast<int32_t*>(take(nb4));
    int32_t* gunit = reinterpret_cast<int32_t*>(take(nb4));
    uint32_t* key = reinterpret_cast<uint32_t*>(take(nb4));
    uint32_t* skey = reinterpret_cast<uint32_t*>(take(nb4));
    uint32_t* snode = reinterpret_cast<uint32_t*>(take(nb4));
    uint8_t* is_input = reinterpret_cast<uint8_t*>(take(align256(nodes)));
    // Per-level unit arrays (units <= inputs <= n): starts, this and the next
    // level's inputs, a scan total.
    void* ubuf = nullptr;
    const size_t un4 = align256(((size_t)n + 2) * 4);
    int st = ctx->alloc(&ubuf, 3 * un4 + 256);
    if (st != ATR_OK) { ctx->release(scratch); return st; }
    char* uq = static_cast<char*>(ubuf);
    uint32_t* ustart = reinterpret_cast<uint32_t*>(uq); uq += un4;
    int32_t* inputs_a = reinterpret_cast<int32_t*>(uq); uq += un4;
    int32_t* inputs_b = reinterpret_cast<int32_t*>(uq); uq += un4;
    uint32_t* d_total = reinterpret_cast<uint32_t*>(uq);

    RefitPlan* plan = new RefitPlan();
    std::vector<void*> level_blocks;
    auto fail = [&](int code) {
        for (void* b : level_blocks) ctx->release(b);
        ctx->release(ubuf);
        ctx->release(scratch);
        delete plan;
        return code;
    };
    auto grid = [](uint64_t work) { return (unsigned)((work + 255) / 256); };

    uint32_t n_inputs = n;
    int32_t* inputs = inputs_a;
    k_plan_leaves<<<grid(n), 256, 0, s>>>(n, inputs);
    ctx->launches += 1;
    for (int level = 0; level < RefitPlan::kMaxLevels; ++level) {
        cudaError_t e = cudaMemsetAsync(cnt, 0, nb4, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(xslot, 0, nb4, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(is_input, 0, align256(nodes), s);
        if (e != cudaSuccess) return fail(cuda_fail(e, "cudaMemsetAsync(refit plan)", __FILE__, __LINE__));
        k_mark_inputs<<<grid(n_inputs), 256, 0, s>>>(inputs, n_inputs, is_input);
        k_plan_count<<<grid(n_inputs), 256, 0, s>>>(t.parent, inputs, n_inputs, cnt, xslot);
        k_plan_roots<<<grid(nodes), 256, 0, s>>>(nodes, t.parent, cnt, flag, size);
        ctx->launches += 3;
        if ((st = exclusive_scan_u32(ctx, flag, uidx, nodes, d_total)) != ATR_OK) return fail(st);
        uint32_t U = 0, total = 0;
        e = cudaMemcpyAsync(&U, d_total, 4, cudaMemcpyDeviceToHost, s);
        if ((st = exclusive_scan_u32(ctx, size, sstart, nodes, d_total)) != ATR_OK) return fail(st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(&total, d_total, 4, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) return fail(cuda_fail(e, "refit plan counts", __FILE__, __LINE__));
        if (total != n_inputs || U == 0) {
            set_error("refit plan: %u units cover %u of %u inputs (the tree's links are not a binary tree)", U, total,
                      n_inputs);
            return fail(ATR_ERR_INVALID_ARG);
        }
        const uint32_t ctas = (total + kUnitInputs - 1) / kUnitInputs;
        const uint32_t n_int = total - U;
        RefitPlan::Level& L = plan->lv[level];
        L.ctas = ctas;
        L.inputs = total;
        L.internal = n_int;
        // Level arrays in one block.
        const size_t c4 = align256(((size_t)ctas + 1) * 4);
        const size_t i4 = align256((size_t)total * 4), i2 = align256((size_t)total * 2);
        const size_t j4 = align256((size_t)(n_int ? n_int : 1) * 4), j2 = align256((size_t)(n_int ? n_int : 1) * 2);
        void* lb = nullptr;
        if ((st = ctx->alloc(&lb, 3 * c4 + 2 * i4 + i2 + 2 * j4 + j2)) != ATR_OK) return fail(st);
        level_blocks.push_back(lb);
        char* lp = static_cast<char*>(lb);
        LevelOut o;
        o.cta_first = reinterpret_cast<uint32_t*>(lp); lp += c4;
        o.cta_in = reinterpret_cast<uint32_t*>(lp); lp += c4;
        o.cta_int = reinterpret_cast<uint32_t*>(lp); lp += c4;
        o.in_src = reinterpret_cast<int32_t*>(lp); lp += i4;
        o.in_node = reinterpret_cast<int32_t*>(lp); lp += i4;
        o.in_par = reinterpret_cast<uint16_t*>(lp); lp += i2;
        o.it_node = reinterpret_cast<int32_t*>(lp); lp += j4;
        o.it_kids = reinterpret_cast<uint32_t*>(lp); lp += j4;
        o.it_par = reinterpret_cast<uint16_t*>(lp);
        L.cta_in = o.cta_in;
        L.cta_int = o.cta_int;
        L.in_src = o.in_src;
        L.in_node = o.in_node;
        L.in_par = o.in_par;
        L.it_node = o.it_node;
        L.it_par = o.it_par;
        L.it_kids = o.it_kids;
        int32_t* next_inputs = inputs == inputs_a ? inputs_b : inputs_a;
        k_plan_units<<<grid(nodes), 256, 0, s>>>(nodes, flag, uidx, sstart, ustart, unit_of, next_inputs);
        k_plan_ctas<<<grid((uint64_t)U + 1), 256, 0, s>>>(U, ctas, ustart, o.cta_first);
        k_plan_cta_offsets<<<grid((uint64_t)ctas + 1), 256, 0, s>>>(U, ctas, total, ustart, o);
        // Slots in node order within each unit (the refit's box stores then
        // go to consecutive nodes): key every unit node, compact in node
        // order, stable sort by key.
        const uint32_t in_units = total + n_int;
        k_plan_keys<<<grid(nodes), 256, 0, s>>>(nodes, t.parent, cnt, flag, is_input, unit_of, key, size);
        if ((st = exclusive_scan_u32(ctx, size, uidx, nodes, nullptr)) != ATR_OK) return fail(st);
        k_plan_compact<<<grid(nodes), 256, 0, s>>>(nodes, size, uidx, key, skey, snode);
        ctx->launches += 5;
        if ((st = atr_device_sort_pairs(ctx, skey, snode, in_units, 32)) != ATR_OK) return fail(st);
        k_plan_slots<<<grid(in_units), 256, 0, s>>>(in_units, skey, snode, ustart, U, total, gslot, gunit);
        k_plan_fill<<<grid(nodes), 256, 0, s>>>(nodes, level, t.parent, t.left, t.right, t.data, cnt, flag, is_input,
                                                gslot, gunit, ustart, o);
        ctx->launches += 2;
        e = cudaGetLastError();
        if (e != cudaSuccess) return fail(cuda_fail(e, "refit plan launch", __FILE__, __LINE__));
        plan->levels = level + 1;
        if (U == 1) break;  // one unit: rooted at the tree's root
        if (level + 1 == RefitPlan::kMaxLevels) return fail(ATR_ERR_UNSUPPORTED);  // too deep a top: no plan
        inputs = next_inputs;
        n_inputs = U;
    }
    cudaError_t e = cudaStreamSynchronize(s);
    ctx->release(ubuf);
    ctx->release(scratch);
    if (e != cudaSuccess) {
        for (void* b : level_blocks) ctx->release(b);
        delete plan;
        return cuda_fail(e, "refit plan", __FILE__, __LINE__);
    }
    plan->blocks = level_blocks;
    *out = plan;
    return ATR_OK;
}

int refit_plan_run(atr_ctx* ctx, const RefitPlan& p, const TreeOut& t, const float4* verts) {
    for (int level = 0; level < p.levels; ++level) {
        const RefitPlan::Level& L = p.lv[level];
        k_refit_level<<<L.ctas, kRefitThreads, kRefitSmem, ctx->stream>>>(level, L.cta_in, L.cta_int, L.in_src, L.in_node,
                                                                 L.in_par, L.it_node, L.it_par, L.it_kids, verts,
                                                                 t.bmin, t.bmax, t.area);
        ctx->launches += 1;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e, "k_refit_level launch", __FILE__, __LINE__);
    return ATR_OK;
}

}  // namespace atr
